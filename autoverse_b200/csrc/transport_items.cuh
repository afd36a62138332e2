// Per-CTA work items of the transport stage (flow: destinations and masses;
// gather: reintegration), shared by the single-world kernels (kernels2d.cu)
// and the batched persistent kernels (batch.cu).
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace flp {

// ---------------------------------------------------------------------------
// Transport in two kernels.
//
// flow_2d (one thread per cell, all channels): channel sum, Sobel of the sum
// and of U_c, alpha, flow, destination dest = x + dt*F (reintegration.rs:81-82)
// and the mass (zeroed below 1e-10, reintegration.rs:76-78), written as three
// planes per channel; it also publishes the largest |dest - x| of any cell
// with mass.
//
// gather_2d (one block per 64x16 tile and channel): with D the largest
// displacement, a source at x overlaps cell ix only if x - ix lies in
// (-(D+s), D+s+1) (reintegration.rs:105-146), so sources x = ix + k with
// k in [-RN, RN+1], RN = ceil(D+s) - 1, cover every deposit.  Each
// destination sums the overlaps of those sources in the reference's deposit
// order (row-major over wrapped source indices), so the result is the
// reference's scatter bit for bit.  No atomics touch the state.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// 16-byte copy (global source and shared destination both 16-byte aligned).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// alpha with the reference's division mass / beta_a; a power-of-two beta_a
// turns it into an exact multiplication.
__device__ __forceinline__ float alpha_fp(float mass, const FlowParams& fp) {
    if (fp.beta_pow2) {
        const float ratio = __fmul_rn(mass, fp.inv_beta);
        float p;
        if (fp.nexp == 1.0f) p = ratio;
        else if (fp.nexp == 2.0f) p = __fmul_rn(ratio, ratio);
        else if (fp.nexp == 3.0f) p = __fmul_rn(__fmul_rn(ratio, ratio), ratio);
        else if (fp.nexp == 4.0f) { const float r2 = __fmul_rn(ratio, ratio); p = __fmul_rn(r2, r2); }
        else p = powf(ratio, fp.nexp);
        if (p < 0.0f) p = 0.0f;  // f32::clamp(0, 1); NaN passes through
        if (p > 1.0f) p = 1.0f;
        return p;
    }
    return flow_alpha(mass, fp.beta_a, fp.nexp);
}

// Window from the largest displacement (dmax slot: float bits of a
// non-negative value; NaN or +inf means unbounded).
__device__ __forceinline__ int window_from_dmax(int bits, const FlowParams& fp, int maxside) {
    const float md = __int_as_float(bits);
    const float rn = ceilf(md + fp.pos_eps + fp.s) - 1.0f;
    const int cap = 2 * maxside + 2;
    if (!(rn < float(cap))) return cap;
    return rn < 0.f ? 0 : int(rn);
}

// Rotated offset order: visits offsets k in [-R, R] so that the wrapped
// coordinates (c + k) mod size come out ascending, which is the order in
// which the reference's row-major scatter deposits into cell c.  Valid when
// 2R+1 <= size; otherwise plain ascending order.
__device__ __forceinline__ int rotated_offset(int j, int c, int R, int size) {
    if (2 * R + 1 > size) return j - R;
    int n_hi = max(0, c + R - (size - 1));
    int n_lo = max(0, R - c);
    if (j < n_hi) return R - n_hi + 1 + j;
    if (j < 2 * R + 1 - n_lo) return -R + n_lo + (j - n_hi);
    return -R + (j - (2 * R + 1 - n_lo));
}

__device__ __forceinline__ int f2i_sat(float v) {
    // Rust `f32 as i32`: saturating, NaN -> 0.
    if (v != v) return 0;
    if (v >= 2147483647.f) return 2147483647;
    if (v <= -2147483648.f) return -2147483647 - 1;
    return int(v);
}

// ------------------------------------------------------------- flow_2d ----
constexpr int FL_W = 32, FL_H = 8;
constexpr int FL_RW = FL_W + 2, FL_RH = FL_H + 2, FL_RC = FL_RW * FL_RH;  // region with the Sobel ring

inline size_t flow_smem_bytes_inl(int C) { return sizeof(float) * (size_t(2 * C + 1) * FL_RC); }

__device__ __forceinline__ void block_max_atomic(float v, bool bad, int* slot) {
    __shared__ float red[32];
    const int anybad = __syncthreads_or(bad ? 1 : 0);
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = red[0];
        for (int w = 1; w < int(blockDim.x >> 5); ++w) m = fmaxf(m, red[w]);
        if (anybad) m = INFINITY;
        if (m > 0.f) atomicMax(slot, __float_as_int(m));  // non-negative floats order like ints
    }
}

// One 32x8 tile of flow_2d; `sm` holds flow_smem_bytes(C).
template <bool POW2>
__device__ void flow_item(float* sm, const float* __restrict__ A, const float* __restrict__ U,
                          float* __restrict__ DX, float* __restrict__ DY, float* __restrict__ MS, int C, int W, int H,
                          const FlowParams& fp, int x0, int y0, int* dmax_slot, int* status) {
    float* as = sm;                    // C staged A planes
    float* us = sm + C * FL_RC;        // C staged U planes
    float* asum = sm + 2 * C * FL_RC;  // channel sum
    __shared__ int colx[FL_RW], rowy[FL_RH];
    const int tid = threadIdx.x;
    const size_t N = size_t(W) * H;
    if (tid < FL_RW) colx[tid] = wrap_near(x0 - 1 + tid, W);
    else if (tid < FL_RW + FL_RH) rowy[tid - FL_RW] = wrap_near(y0 - 1 + (tid - FL_RW), H);
    __syncthreads();
    for (int i = tid; i < 2 * C * FL_RC; i += 256) {
        const int k = i / FL_RC, cell = i - k * FL_RC;
        const int ly = cell / FL_RW, lx = cell - ly * FL_RW;
        const size_t idx = size_t(rowy[ly]) * W + colx[lx];
        cp_async4(sm + i, (k < C ? A + size_t(k) * N : U + size_t(k - C) * N) + idx);
    }
    cp_async_wait_all();
    __syncthreads();
    for (int i = tid; i < FL_RC; i += 256) {
        float a = 0.f;
        for (int k = 0; k < C; ++k) a = __fadd_rn(a, as[k * FL_RC + i]);
        asum[i] = a;
    }
    __syncthreads();
    const int lx = tid & (FL_W - 1), ly = tid / FL_W;
    const int X = x0 + lx, Y = y0 + ly;
    float dmax = 0.f;
    bool bad = false;
    if (X < W && Y < H) {
        const int o = ly * FL_RW + lx;  // top-left of the 3x3 window
        const float* a = asum + o;
        float gax, gay;
        sobel2(a[0], a[1], a[2], a[FL_RW], a[FL_RW + 2], a[2 * FL_RW], a[2 * FL_RW + 1], a[2 * FL_RW + 2], gax, gay);
        const float alpha = alpha_fp(a[FL_RW + 1], fp);
        const float oma = __fsub_rn(1.0f, alpha);
        const float agx = __fmul_rn(alpha, gax), agy = __fmul_rn(alpha, gay);
        const size_t cell = size_t(Y) * W + X;
        for (int c = 0; c < C; ++c) {
            const float* u = us + c * FL_RC + o;
            float gux, guy;
            sobel2(u[0], u[1], u[2], u[FL_RW], u[FL_RW + 2], u[2 * FL_RW], u[2 * FL_RW + 1], u[2 * FL_RW + 2], gux,
                   guy);
            const float fx = __fsub_rn(__fmul_rn(oma, gux), agx);
            const float fy = __fsub_rn(__fmul_rn(oma, guy), agy);
            const float dx = __fadd_rn(float(X), __fmul_rn(fp.dt, fx));
            const float dy = __fadd_rn(float(Y), __fmul_rn(fp.dt, fy));
            float mass = as[c * FL_RC + o + FL_RW + 1];
            bad |= !(isfinite(mass) && isfinite(dx) && isfinite(dy));
            if (fabsf(mass) < 1e-10f) mass = 0.f;
            if (mass != 0.f) dmax = fmaxf(dmax, fmaxf(fabsf(dx - float(X)), fabsf(dy - float(Y))));
            DX[size_t(c) * N + cell] = dx;
            DY[size_t(c) * N + cell] = dy;
            MS[size_t(c) * N + cell] = POW2 ? __fmul_rn(mass, fp.inv_area) : mass;
        }
    }
    if (status && __syncthreads_or(bad ? 1 : 0) && tid == 0) atomicOr(status, STATUS_NONFINITE);
    block_max_atomic(dmax, bad, dmax_slot);
    __syncthreads();
}

// ------------------------------------------------- flow_2d, row-walking ----
// Register-resident variant for C <= 4 (same arithmetic as flow_item): a warp
// covers 32 columns and each thread walks FR_RPT rows of its column, keeping a
// 3-row window of the channel sum and of every U_c in registers.  Horizontal
// neighbours come from warp shuffles; the two columns just outside the warp
// (x0-1 for lane 0, x0+32 for lane 31) from one extra load per row and field.
// Every lane loads the wrapped column of its position, so partial tiles and
// grids narrower than a warp see the torus neighbours.
constexpr int FR_RPT = 2;            // rows per thread
constexpr int FR_H = 8 * FR_RPT;     // tile height: 8 warps of 32 columns

template <int C, bool POW2>
__device__ __forceinline__ void flow_rows_item(const float* __restrict__ A, const float* __restrict__ U,
                                               float* __restrict__ DX, float* __restrict__ DY,
                                               float* __restrict__ MS, int W, int H, const FlowParams& fp, int x0,
                                               int y0, int* dmax_slot, int* status) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const size_t N = size_t(W) * H;
    const int X = x0 + lane;
    const int xc = wrap_near(X, W);
    const int xh = wrap_near(lane == 0 ? x0 - 1 : x0 + 32, W);
    const int yb = y0 + FR_RPT * wp;
    float sw[3][3], uw[C][3][3], ac[C], an[C];
    float dmax = 0.f;
    bool bad = false;
#pragma unroll
    for (int r = 0; r < FR_RPT + 2; ++r) {
        const size_t row = size_t(wrap_near(yb - 1 + r, H)) * W;
        float av[C], ah[C], uv[C], uh[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            av[c] = A[size_t(c) * N + row + xc];
            ah[c] = A[size_t(c) * N + row + xh];
            uv[c] = U[size_t(c) * N + row + xc];
            uh[c] = U[size_t(c) * N + row + xh];
        }
        float sv = 0.f, sh = 0.f;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            sv = __fadd_rn(sv, av[c]);
            sh = __fadd_rn(sh, ah[c]);
        }
        // shift the windows up one row
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            sw[0][j] = sw[1][j];
            sw[1][j] = sw[2][j];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                uw[c][0][j] = uw[c][1][j];
                uw[c][1][j] = uw[c][2][j];
            }
        }
        {
            const float l = __shfl_up_sync(FULL, sv, 1), rr = __shfl_down_sync(FULL, sv, 1);
            sw[2][0] = lane == 0 ? sh : l;
            sw[2][1] = sv;
            sw[2][2] = lane == 31 ? sh : rr;
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const float l = __shfl_up_sync(FULL, uv[c], 1), rr = __shfl_down_sync(FULL, uv[c], 1);
            uw[c][2][0] = lane == 0 ? uh[c] : l;
            uw[c][2][1] = uv[c];
            uw[c][2][2] = lane == 31 ? uh[c] : rr;
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
            ac[c] = an[c];  // A_c of the window's centre row
            an[c] = av[c];
        }
        if (r < 2) continue;
        const int Y = yb + r - 2;
        if (X >= W || Y >= H) continue;
        float gax, gay;
        sobel2(sw[0][0], sw[0][1], sw[0][2], sw[1][0], sw[1][2], sw[2][0], sw[2][1], sw[2][2], gax, gay);
        const float alpha = alpha_fp(sw[1][1], fp);
        const float oma = __fsub_rn(1.0f, alpha);
        const float agx = __fmul_rn(alpha, gax), agy = __fmul_rn(alpha, gay);
        const size_t cell = size_t(Y) * W + X;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            float gux, guy;
            sobel2(uw[c][0][0], uw[c][0][1], uw[c][0][2], uw[c][1][0], uw[c][1][2], uw[c][2][0], uw[c][2][1],
                   uw[c][2][2], gux, guy);
            const float fx = __fsub_rn(__fmul_rn(oma, gux), agx);
            const float fy = __fsub_rn(__fmul_rn(oma, guy), agy);
            const float dx = __fadd_rn(float(X), __fmul_rn(fp.dt, fx));
            const float dy = __fadd_rn(float(Y), __fmul_rn(fp.dt, fy));
            float mass = ac[c];
            bad |= !(isfinite(mass) && isfinite(dx) && isfinite(dy));
            if (fabsf(mass) < 1e-10f) mass = 0.f;
            if (mass != 0.f) dmax = fmaxf(dmax, fmaxf(fabsf(dx - float(X)), fabsf(dy - float(Y))));
            DX[size_t(c) * N + cell] = dx;
            DY[size_t(c) * N + cell] = dy;
            MS[size_t(c) * N + cell] = POW2 ? __fmul_rn(mass, fp.inv_area) : mass;
        }
    }
    if (status && __syncthreads_or(bad ? 1 : 0) && threadIdx.x == 0) atomicOr(status, STATUS_NONFINITE);
    block_max_atomic(dmax, bad, dmax_slot);
}

// ----------------------------------------------------------- gather_2d ----
constexpr int GT_W = 64, GT_H = 16, TP = 4, RN_MAX = 3;
// Staged source columns: x0 - TP .. x0 + GT_W + TP - 1 plus 4 unused ones, so
// that a row is 76 floats: with the column-major thread mapping of the gather
// (a warp is 2 x 16 threads, 16 rows apart) the rows of a quarter-warp then
// start in distinct bank groups.
constexpr int SR_W = GT_W + 2 * TP + 4;
constexpr int SR_HMAX = GT_H + 2 * RN_MAX + 1;  // up to 23 source rows
static_assert(SR_W % 4 == 0, "source rows must stay 16-byte aligned");

inline size_t gather_smem_bytes_inl() { return sizeof(float) * 5 * SR_W * SR_HMAX; }

// Stage the dx, dy and m planes of an SR_W x SRH source region (columns
// colx[], rows rowy[]) into shared memory.  When W and the three base
// pointers allow it, whole 16-byte chunks are copied: x0 - TP and W are
// multiples of 4, so every chunk of 4 source columns is 4 contiguous, aligned
// columns after the wrap.
template <int SRH, int SW>
__device__ __forceinline__ void stage_sources(float* sdx, float* sdy, float* smass, const float* __restrict__ DX,
                                              const float* __restrict__ DY, const float* __restrict__ MS,
                                              const int* colx, const int* rowy, int W) {
    const int tid = threadIdx.x;
    const bool vec = (W & 3) == 0 &&
                     ((reinterpret_cast<uintptr_t>(DX) | reinterpret_cast<uintptr_t>(DY) |
                       reinterpret_cast<uintptr_t>(MS)) & 15) == 0;
    if (vec) {
        constexpr int CH = SW / 4;
        for (int i = tid; i < 3 * SRH * CH; i += 256) {
            const int k = i / (SRH * CH), rem = i - k * (SRH * CH);
            const int sy = rem / CH, c4 = rem - sy * CH;
            const size_t idx = size_t(rowy[sy]) * W + colx[4 * c4];
            const int cell = sy * SW + 4 * c4;
            float* dst = k == 0 ? sdx + cell : (k == 1 ? sdy + cell : smass + cell);
            cp_async16(dst, (k == 0 ? DX : (k == 1 ? DY : MS)) + idx);
        }
    } else {
        constexpr int NS = SW * SRH;
        for (int i = tid; i < 3 * NS; i += 256) {
            const int k = i / NS, cell = i - k * NS;
            const int sy = cell / SW, sx = cell - sy * SW;
            const size_t idx = size_t(rowy[sy]) * W + colx[sx];
            float* dst = k == 0 ? sdx + cell : (k == 1 ? sdy + cell : smass + cell);
            cp_async4(dst, (k == 0 ? DX : (k == 1 ? DY : MS)) + idx);
        }
    }
}

__device__ __forceinline__ int wrap_pass(int g, int size) { return g >= size ? 0 : (g < 0 ? 2 : 1); }

// Whether a gather tile uses the column-major thread mapping: tiles whose
// sources reach across an x edge of the torus.  Each thread takes the wrap
// passes of its own window, and with this mapping the threads that need more
// than one pass sit in the two edge warps instead of in every warp.
__device__ __forceinline__ bool gather_column_major(int x0, int W, int RN) {
    return x0 - RN < 0 || x0 + GT_W + RN >= W;
}

// One source row of the gather for the thread's 4 destinations X0..X0+3.
// Source column j of the strip window is x0-TP+4tx+j; its offset from
// destination i is kx = j - TP - i, kept in [-RN, RN+1] at compile time.
// Sources are streamed one float4 chunk (4 columns) at a time.  CHECK adds
// the wrap-pass predicate for tiles whose source columns wrap the torus.
template <int RN, bool POW2, bool CHECK>
__device__ __forceinline__ void gather_row(const float* __restrict__ rxmin, const float* __restrict__ rxmax,
                                           const float* __restrict__ rymin, const float* __restrict__ rymax,
                                           const float* __restrict__ rm, float cy0, float cy1, int X0, int gx_base,
                                           int W, int cp, float total_area, float (&acc)[4]) {
    constexpr int JLO = TP - RN, JHI = TP + 3 + RN + 1;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        if (4 * q + 3 < JLO || 4 * q > JHI) continue;
        const float4 vxa = *reinterpret_cast<const float4*>(rxmin + 4 * q);
        const float4 vxb = *reinterpret_cast<const float4*>(rxmax + 4 * q);
        const float4 vya = *reinterpret_cast<const float4*>(rymin + 4 * q);
        const float4 vyb = *reinterpret_cast<const float4*>(rymax + 4 * q);
        const float4 vm = *reinterpret_cast<const float4*>(rm + 4 * q);
        const float xa[4] = {vxa.x, vxa.y, vxa.z, vxa.w}, xb[4] = {vxb.x, vxb.y, vxb.z, vxb.w};
        const float ya[4] = {vya.x, vya.y, vya.z, vya.w}, yb[4] = {vyb.x, vyb.y, vyb.z, vyb.w};
        const float mm[4] = {vm.x, vm.y, vm.z, vm.w};
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int j = 4 * q + jj;
            if (j < JLO || j > JHI) continue;
            int xsh = 0;
            if (CHECK) {
                const int gx = gx_base + j;
                if (wrap_pass(gx, W) != cp) continue;
                xsh = gx < 0 ? W : (gx >= W ? -W : 0);
            }
            const float m = mm[jj];
            const float oy0 = fmaxf(cy0, ya[jj]), oy1 = fminf(cy1, yb[jj]);
            const float oh = fmaxf(__fsub_rn(oy1, oy0), 0.f);
            // POW2: a zero mass or a zero height adds a signed zero, which
            // leaves acc (never -0: it starts at +0) unchanged, so the loop
            // runs branch-free; the division path keeps the reference's skip.
            if (!POW2 && (m == 0.f || !(oh > 0.f))) continue;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (j - TP - i < -RN || j - TP - i > RN + 1) continue;
                const int ix = X0 + i + xsh;
                const float ox0 = fmaxf(float(ix), xa[jj]), ox1 = fminf(float(ix + 1), xb[jj]);
                const float ow = fmaxf(__fsub_rn(ox1, ox0), 0.f);
                const float area = __fmul_rn(ow, oh);
                if (POW2) {
                    // m holds mass * (1 / total_area), exact for a power-of-two
                    // area; a zero area adds a signed zero, which leaves acc as is.
                    acc[i] = __fadd_rn(acc[i], __fmul_rn(m, area));
                } else if (area > 0.f) {
                    acc[i] = __fadd_rn(acc[i], __fmul_rn(m, __fdiv_rn(area, total_area)));
                }
            }
        }
    }
}

template <int RN, bool POW2>
__device__ __forceinline__ void gather_strip(const float* sxmin, const float* sxmax, const float* symin,
                                             const float* symax, const float* smass, float* __restrict__ out, int W,
                                             int H, const FlowParams& fp, int x0, int y0, int sw, float (&acc)[4]) {
    // Tiles at an x edge of the torus use the column-major mapping (a warp owns
    // 2 columns of 4 destinations x 16 rows), so only the two warps at the
    // edge take the wrap-pass path; other tiles map a warp to 2 rows.
    const bool cm = gather_column_major(x0, W, RN);
    const int tx = cm ? threadIdx.x >> 4 : threadIdx.x & 15, ty = cm ? threadIdx.x & 15 : threadIdx.x >> 4;
    const int Y = y0 + ty, X0 = x0 + 4 * tx;
    // wrap passes of this thread's own window (sources X0-RN .. X0+4+RN, Y-RN .. Y+RN+1)
    const int rp_lo = (Y + RN + 1 >= H) ? 0 : 1, rp_hi = (Y - RN < 0) ? 2 : 1;
    const int cp_lo = (X0 + 4 + RN >= W) ? 0 : 1, cp_hi = (X0 - RN < 0) ? 2 : 1;
    const bool xin = cp_lo == 1 && cp_hi == 1;
    const int gx_base = x0 - TP + 4 * tx;
    for (int rp = rp_lo; rp <= rp_hi; ++rp) {
#pragma unroll 1
        for (int ky = -RN; ky <= RN + 1; ++ky) {
            const int gy = Y + ky;
            if (wrap_pass(gy, H) != rp) continue;
            const int iy = Y + (gy < 0 ? H : (gy >= H ? -H : 0));
            const float cy0 = float(iy), cy1 = float(iy + 1);
            const int off = (ty + RN + ky) * sw + 4 * tx;
            if (xin) {
                gather_row<RN, POW2, false>(sxmin + off, sxmax + off, symin + off, symax + off, smass + off, cy0,
                                            cy1, X0, gx_base, W, 1, fp.total_area, acc);
            } else {
                for (int cp = cp_lo; cp <= cp_hi; ++cp)
                    gather_row<RN, POW2, true>(sxmin + off, sxmax + off, symin + off, symax + off, smass + off,
                                               cy0, cy1, X0, gx_base, W, cp, fp.total_area, acc);
            }
        }
    }
    float* o = out + size_t(Y) * W;
    if (X0 + 3 < W && (W & 3) == 0) {
        *reinterpret_cast<float4*>(o + X0) = make_float4(acc[0], acc[1], acc[2], acc[3]);
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (X0 + i < W) o[X0 + i] = acc[i];
    }
}

template <int RN, bool POW2>
__device__ void gather_body(float* sm, const float* __restrict__ DX, const float* __restrict__ DY,
                            const float* __restrict__ MS, float* __restrict__ out, int W, int H, const FlowParams& fp,
                            int x0, int y0, float (&acc)[4]) {
    constexpr int SRH = GT_H + 2 * RN + 1;
    const int tid = threadIdx.x;
    const bool cm = gather_column_major(x0, W, RN);
    const int tx = cm ? tid >> 4 : tid & 15, ty = cm ? tid & 15 : tid >> 4;
    const int sw = cm ? SR_W : SR_W - 4;  // row stride: padded only for the column-major mapping
    float* sxmin = sm;                    // SRH x sw each
    float* sxmax = sxmin + sw * SRH;
    float* symin = sxmax + sw * SRH;
    float* symax = symin + sw * SRH;
    float* smass = symax + sw * SRH;
    __shared__ int colx[SR_W], rowy[SRH];
    const float s = fp.s;
    if (tid < SR_W) colx[tid] = wrap_near(x0 - TP + tid, W);
    else if (tid < SR_W + SRH) rowy[tid - SR_W] = wrap_near(y0 - RN + (tid - SR_W), H);
    __syncthreads();
    // stage destinations and masses (dx -> xmin in place, dy -> ymin in place)
    if (cm) stage_sources<SRH, SR_W>(sxmin, symin, smass, DX, DY, MS, colx, rowy, W);
    else stage_sources<SRH, SR_W - 4>(sxmin, symin, smass, DX, DY, MS, colx, rowy, W);
    cp_async_wait_all();
    __syncthreads();
    for (int i = 4 * tid; i < sw * SRH; i += 1024) {
        const float4 dx = *reinterpret_cast<const float4*>(sxmin + i);
        const float4 dy = *reinterpret_cast<const float4*>(symin + i);
        *reinterpret_cast<float4*>(sxmin + i) =
            make_float4(__fsub_rn(dx.x, s), __fsub_rn(dx.y, s), __fsub_rn(dx.z, s), __fsub_rn(dx.w, s));
        *reinterpret_cast<float4*>(sxmax + i) =
            make_float4(__fadd_rn(dx.x, s), __fadd_rn(dx.y, s), __fadd_rn(dx.z, s), __fadd_rn(dx.w, s));
        *reinterpret_cast<float4*>(symin + i) =
            make_float4(__fsub_rn(dy.x, s), __fsub_rn(dy.y, s), __fsub_rn(dy.z, s), __fsub_rn(dy.w, s));
        *reinterpret_cast<float4*>(symax + i) =
            make_float4(__fadd_rn(dy.x, s), __fadd_rn(dy.y, s), __fadd_rn(dy.z, s), __fadd_rn(dy.w, s));
    }
    __syncthreads();
    const int Y = y0 + ty, X0 = x0 + 4 * tx;
    if (Y < H && X0 < W)
        gather_strip<RN, POW2>(sxmin, sxmax, symin, symax, smass, out, W, H, fp, x0, y0, sw, acc);
    __syncthreads();
}

// Reintegrated mass at destination (X, Y) for any window, sources read from
// the destination planes in global memory.  Handles the nearest-cell mode,
// the reference's [-W, 2W] cell clamp, and windows wider than the grid.
template <bool POW2>
__device__ float gather_generic_2d(const float* __restrict__ DX, const float* __restrict__ DY,
                                   const float* __restrict__ MS, int W, int H, int X, int Y, int R,
                                   const FlowParams& fp) {
    float acc = 0.f;
    for (int jy = 0; jy <= 2 * R; ++jy) {
        const int ky = rotated_offset(jy, Y, R, H);
        const int yw = wrap_coord(Y + ky, H);
        const int iy = yw - ky;
        for (int jx = 0; jx <= 2 * R; ++jx) {
            const int kx = rotated_offset(jx, X, R, W);
            const int xw = wrap_coord(X + kx, W);
            const int ix = xw - kx;
            const size_t src = size_t(yw) * W + xw;
            const float m = MS[src];
            if (m == 0.f) continue;
            const float dx = DX[src], dy = DY[src];
            if (fp.point_mode) {
                if (f2i_sat(roundf(dx)) == ix && f2i_sat(roundf(dy)) == iy) acc = __fadd_rn(acc, m);
                continue;
            }
            const float xmin = __fsub_rn(dx, fp.s), xmax = __fadd_rn(dx, fp.s);
            const float ymin = __fsub_rn(dy, fp.s), ymax = __fadd_rn(dy, fp.s);
            const int ix_lo = max(f2i_sat(floorf(xmin)), -W), ix_hi = min(f2i_sat(ceilf(xmax)), 2 * W);
            const int iy_lo = max(f2i_sat(floorf(ymin)), -H), iy_hi = min(f2i_sat(ceilf(ymax)), 2 * H);
            if (ix < ix_lo || ix > ix_hi || iy < iy_lo || iy > iy_hi) continue;
            const float ox0 = fmaxf(float(ix), xmin), ox1 = fminf(float(ix + 1), xmax);
            const float oy0 = fmaxf(float(iy), ymin), oy1 = fminf(float(iy + 1), ymax);
            const float ow = fmaxf(__fsub_rn(ox1, ox0), 0.f);
            const float oh = fmaxf(__fsub_rn(oy1, oy0), 0.f);
            const float area = __fmul_rn(ow, oh);
            if (!(area > 0.f)) continue;
            acc = __fadd_rn(acc, POW2 ? __fmul_rn(m, area) : __fmul_rn(m, __fdiv_rn(area, fp.total_area)));
        }
    }
    return acc;
}

// One 64x16 tile of one channel of gather_2d; `sm` holds gather_smem_bytes().
// dxc/dyc/msc/out are that channel's planes.
template <bool POW2>
__device__ void gather_item(float* sm, const float* __restrict__ dxc, const float* __restrict__ dyc,
                            const float* __restrict__ msc, float* __restrict__ out, int W, int H,
                            const FlowParams& fp, int dmax_bits, int x0, int y0) {
    const int RN = window_from_dmax(dmax_bits, fp, max(W, H));
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    const bool fast = RN <= RN_MAX && 2 * RN + 2 <= W && 2 * RN + 2 <= H && !fp.point_mode;
    if (fast) {
        switch (RN) {
            case 0: gather_body<0, POW2>(sm, dxc, dyc, msc, out, W, H, fp, x0, y0, acc); break;
            case 1: gather_body<1, POW2>(sm, dxc, dyc, msc, out, W, H, fp, x0, y0, acc); break;
            case 2: gather_body<2, POW2>(sm, dxc, dyc, msc, out, W, H, fp, x0, y0, acc); break;
            default: gather_body<3, POW2>(sm, dxc, dyc, msc, out, W, H, fp, x0, y0, acc); break;
        }
        return;
    }
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int Y = y0 + ty;
#pragma unroll 1
    for (int i = 0; i < 4; ++i) {
        const int X = x0 + 4 * tx + i;
        if (X < W && Y < H) out[size_t(Y) * W + X] = gather_generic_2d<POW2>(dxc, dyc, msc, W, H, X, Y, RN + 1, fp);
    }
}


}  // namespace flp
