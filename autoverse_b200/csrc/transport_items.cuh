// Per-CTA work items of the transport stage (flow: destinations and masses;
// gather: reintegration), shared by the single-world kernels (kernels2d.cu)
// and the batched persistent kernels (batch.cu).
#pragma once

#include "common.cuh"
#include "kernels.h"

#include <type_traits>


namespace flp {

// ---------------------------------------------------------------------------
// Transport in two kernels.
//
// flow_2d (one thread per cell, all channels): channel sum, Sobel of the sum
// and of U_c, alpha, flow and destination dest = x + dt*F
// (reintegration.rs:81-82), written as two planes per channel; it also
// publishes the largest |dest - x| of any cell with mass.  The gather takes a
// source's mass from the state itself (source_mass: zero below 1e-10,
// reintegration.rs:76-78).
//
// gather_2d (one block per 64x16 or 64x32 tile and channel, 4x1 or 4x2
// destinations per thread): with D the largest
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
// turns it into an exact multiplication.  T = float in the engine, double in
// the FP64 twin (the parameters are the f32 values the reference uses).
template <class T>
__device__ __forceinline__ T alpha_fp(T mass, const FlowParams& fp) {
    if (fp.beta_pow2) {
        const T ratio = rn_mul(mass, T(fp.inv_beta));
        T p;
        if (fp.nexp == 1.0f) p = ratio;
        else if (fp.nexp == 2.0f) p = rn_mul(ratio, ratio);
        else if (fp.nexp == 3.0f) p = rn_mul(rn_mul(ratio, ratio), ratio);
        else if (fp.nexp == 4.0f) { const T r2 = rn_mul(ratio, ratio); p = rn_mul(r2, r2); }
        else p = r_pow(ratio, T(fp.nexp));
        if (p < T(0)) p = T(0);  // f32::clamp(0, 1); NaN passes through
        if (p > T(1)) p = T(1);
        return p;
    }
    return flow_alpha(mass, T(fp.beta_a), T(fp.nexp));
}

// Per-cell flow (propagator.rs:304-330, flow.rs:68-87) and destination
// (reintegration.rs:81-82), shared by every flow kernel: flow_mix takes the
// 3x3 window of the channel sum, flow_destination the 3x3 window of one U_c.
template <class T>
struct FlowMix {
    T oma, agx, agy;  // 1 - alpha, alpha * grad(sum)
};
template <class T>
__device__ __forceinline__ FlowMix<T> flow_mix(T tl, T tc, T tr, T ml, T mc, T mr, T bl, T bc, T br,
                                               const FlowParams& fp) {
    T gax, gay;
    sobel2(tl, tc, tr, ml, mr, bl, bc, br, gax, gay);
    const T alpha = alpha_fp(mc, fp);
    return {rn_sub(T(1), alpha), rn_mul(alpha, gax), rn_mul(alpha, gay)};
}
template <class T>
__device__ __forceinline__ void flow_destination(const FlowMix<T>& f, T tl, T tc, T tr, T ml, T mr, T bl, T bc,
                                                 T br, int X, int Y, const FlowParams& fp, T& dx, T& dy) {
    T gux, guy;
    sobel2(tl, tc, tr, ml, mr, bl, bc, br, gux, guy);
    const T fx = rn_sub(rn_mul(f.oma, gux), f.agx);
    const T fy = rn_sub(rn_mul(f.oma, guy), f.agy);
    dx = rn_add(T(X), rn_mul(T(fp.dt), fx));
    dy = rn_add(T(Y), rn_mul(T(fp.dt), fy));
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

template <class T>
__device__ __forceinline__ int f2i_sat(T v) {
    // Rust `f32 as i32`: saturating, NaN -> 0.
    if (v != v) return 0;
    if (v >= T(2147483647.f)) return 2147483647;
    if (v <= T(-2147483648.f)) return -2147483647 - 1;
    return int(v);
}

// The mass a source at state value a deposits: zero below the reference's
// 1e-10 threshold (reintegration.rs:76-78), pre-scaled by 1/(2s)^2 when that
// factor is a power of two (then m * area equals the reference's
// mass * (area / total_area) exactly).
template <bool POW2, class T>
__device__ __forceinline__ T source_mass(T a, const FlowParams& fp) {
    const T m = fabs(a) < T(1e-10f) ? T(0) : a;
    return POW2 ? rn_mul(m, T(fp.inv_area)) : m;
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
inline __device__ void flow_item(float* sm, const float* __restrict__ A, const float* __restrict__ U,
                                 float* __restrict__ DX, float* __restrict__ DY, int C, int W, int H,
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
        const FlowMix<float> f = flow_mix(a[0], a[1], a[2], a[FL_RW], a[FL_RW + 1], a[FL_RW + 2], a[2 * FL_RW],
                                          a[2 * FL_RW + 1], a[2 * FL_RW + 2], fp);
        const size_t cell = size_t(Y) * W + X;
        for (int c = 0; c < C; ++c) {
            const float* u = us + c * FL_RC + o;
            float dx, dy;
            flow_destination(f, u[0], u[1], u[2], u[FL_RW], u[FL_RW + 2], u[2 * FL_RW], u[2 * FL_RW + 1],
                             u[2 * FL_RW + 2], X, Y, fp, dx, dy);
            const float mass = as[c * FL_RC + o + FL_RW + 1];
            bad |= !(isfinite(mass) && isfinite(dx) && isfinite(dy));
            if (fabsf(mass) >= 1e-10f) dmax = fmaxf(dmax, fmaxf(fabsf(dx - float(X)), fabsf(dy - float(Y))));
            DX[size_t(c) * N + cell] = dx;
            DY[size_t(c) * N + cell] = dy;
        }
    }
    if (status && __syncthreads_or(bad ? 1 : 0) && tid == 0) atomicOr(status, STATUS_NONFINITE);
    block_max_atomic(dmax, bad, dmax_slot);
    __syncthreads();
}

// ------------------------------------------------- flow_2d, row-walking ----
// Register-resident variant for C <= 4 (same arithmetic as flow_item): a warp
// covers 32 columns and each thread walks RPT rows of its column, keeping a
// 3-row window of the channel sum and of every U_c in registers.  Horizontal
// neighbours come from warp shuffles; the two columns just outside the warp
// (x0-1 for lane 0, x0+32 for lane 31) from one extra load per row and field.
// Every lane loads the wrapped column of its position, so partial tiles and
// grids narrower than a warp see the torus neighbours.
#ifndef FLP_FR_RPT
#define FLP_FR_RPT 2
#endif
constexpr int FR_RPT = FLP_FR_RPT;   // rows per thread of the single-world kernels
constexpr int FR_H = 8 * FR_RPT;     // tile height: 8 warps of 32 columns

template <int C, int RPT = FR_RPT>
__device__ __forceinline__ void flow_rows_item(const float* __restrict__ A, const float* __restrict__ U,
                                               float* __restrict__ DX, float* __restrict__ DY, int W, int H,
                                               const FlowParams& fp, int x0, int y0, int* dmax_slot, int* status) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const size_t N = size_t(W) * H;
    const int X = x0 + lane;
    const int xc = wrap_near(X, W);
    const int xh = wrap_near(lane == 0 ? x0 - 1 : x0 + 32, W);
    const int yb = y0 + RPT * wp;
    float sw[3][3], uw[C][3][3], ac[C], an[C];
    float dmax = 0.f;
    bool bad = false;
#pragma unroll
    for (int r = 0; r < RPT + 2; ++r) {
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
        const FlowMix<float> f = flow_mix(sw[0][0], sw[0][1], sw[0][2], sw[1][0], sw[1][1], sw[1][2], sw[2][0],
                                          sw[2][1], sw[2][2], fp);
        const size_t cell = size_t(Y) * W + X;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            float dx, dy;
            flow_destination(f, uw[c][0][0], uw[c][0][1], uw[c][0][2], uw[c][1][0], uw[c][1][2], uw[c][2][0],
                             uw[c][2][1], uw[c][2][2], X, Y, fp, dx, dy);
            const float mass = ac[c];
            bad |= !(isfinite(mass) && isfinite(dx) && isfinite(dy));
            if (fabsf(mass) >= 1e-10f) dmax = fmaxf(dmax, fmaxf(fabsf(dx - float(X)), fabsf(dy - float(Y))));
            DX[size_t(c) * N + cell] = dx;
            DY[size_t(c) * N + cell] = dy;
        }
    }
    if (status && __syncthreads_or(bad ? 1 : 0) && threadIdx.x == 0) atomicOr(status, STATUS_NONFINITE);
    block_max_atomic(dmax, bad, dmax_slot);
}

// ----------------------------------------------------------- gather_2d ----
// A tile is 64 x (16 * GBY) destinations; each of its 256 threads sums a
// block of 4 x GBY destinations, so a source's x overlaps serve GBY rows and
// its y overlaps serve 4 columns.  The single-world kernel uses GBY = 1 (its
// one wave of tiles then overlaps staging and compute across co-resident
// blocks); the batched engine, whose persistent blocks pull tiles from a
// queue, uses GBY = 2.
constexpr int GT_W = 64, TP = 4, RN_MAX = 3;
__host__ __device__ constexpr int gt_h(int gby) { return 16 * gby; }
// Staged source columns: x0 - TP .. x0 + GT_W + TP - 1 plus 4 unused ones, so
// that a row is 76 floats: with the column-major thread mappings of the
// gather (gather_thread) the rows of a quarter-warp then start in distinct
// bank groups.
constexpr int SR_W = GT_W + 2 * TP + 4;
__host__ __device__ constexpr int sr_hmax(int gby) { return gt_h(gby) + 2 * RN_MAX + 1; }  // up to 39 source rows
static_assert(SR_W % 4 == 0, "source rows must stay 16-byte aligned");

inline size_t gather_smem_bytes_inl(int gby) { return sizeof(float) * 5 * SR_W * sr_hmax(gby); }

// Stage the dx, dy and state planes of an SR_W x SRH source region (columns
// colx[], rows rowy[]) into shared memory.  When W and the three base
// pointers allow it, whole 16-byte chunks are copied: x0 - TP and W are
// multiples of 4, so every chunk of 4 source columns is 4 contiguous, aligned
// columns after the wrap.
template <int SRH, int SW>
__device__ __forceinline__ void stage_sources(float* sdx, float* sdy, float* smass, const float* __restrict__ DX,
                                              const float* __restrict__ DY, const float* __restrict__ AS,
                                              const int* colx, const int* rowy, int W) {
    const int tid = threadIdx.x;
    const bool vec = (W & 3) == 0 &&
                     ((reinterpret_cast<uintptr_t>(DX) | reinterpret_cast<uintptr_t>(DY) |
                       reinterpret_cast<uintptr_t>(AS)) & 15) == 0;
    if (vec) {
        constexpr int CH = SW / 4;
        for (int i = tid; i < 3 * SRH * CH; i += 256) {
            const int k = i / (SRH * CH), rem = i - k * (SRH * CH);
            const int sy = rem / CH, c4 = rem - sy * CH;
            const size_t idx = size_t(rowy[sy]) * W + colx[4 * c4];
            const int cell = sy * SW + 4 * c4;
            float* dst = k == 0 ? sdx + cell : (k == 1 ? sdy + cell : smass + cell);
            cp_async16(dst, (k == 0 ? DX : (k == 1 ? DY : AS)) + idx);
        }
    } else {
        constexpr int NS = SW * SRH;
        for (int i = tid; i < 3 * NS; i += 256) {
            const int k = i / NS, cell = i - k * NS;
            const int sy = cell / SW, sx = cell - sy * SW;
            const size_t idx = size_t(rowy[sy]) * W + colx[sx];
            float* dst = k == 0 ? sdx + cell : (k == 1 ? sdy + cell : smass + cell);
            cp_async4(dst, (k == 0 ? DX : (k == 1 ? DY : AS)) + idx);
        }
    }
}

__device__ __forceinline__ int wrap_pass(int g, int size) { return g >= size ? 0 : (g < 0 ? 2 : 1); }

// a - b rounded to nearest, then clamped to [0, 1] (one instruction).
__device__ __forceinline__ float fsub_sat(float a, float b) {
    float d;
    asm("sub.rn.sat.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}

// Overlap of the unit cell [c0, c0 + 1) (c1 = c0 + 1, both integers) with a
// source square's side [lo, hi]: the reference's max(min(c1, hi) - max(c0, lo),
// 0) (reintegration.rs:119-126).  WIDE (hi - lo >= 1.5 before rounding, so
// hi - lo > 1 after it): the square cannot lie inside the cell, and the
// overlap is min(sat(hi - c0), sat(c1 - lo)) with the same single rounding in
// every case: a side that ends inside the cell gives the reference's one
// subtraction, a side beyond it saturates to 1, a side short of it to 0.  That
// form takes two FMA-pipe subtractions and one min instead of three min/max
// and a subtraction.
template <bool WIDE>
__device__ __forceinline__ float cell_overlap(float c0, float c1, float lo, float hi) {
    if (WIDE) return fminf(fsub_sat(hi, c0), fsub_sat(c1, lo));
    return fmaxf(__fsub_rn(fminf(c1, hi), fmaxf(c0, lo)), 0.f);
}

// Whether a gather tile uses the column-major thread mapping: tiles whose
// sources reach across an x edge of the torus.  Each thread takes the wrap
// passes of its own window, and with this mapping the threads that need more
// than one pass sit in the two edge warps instead of in every warp.
__device__ __forceinline__ bool gather_column_major(int x0, int W, int RN) {
    return x0 - RN < 0 || x0 + GT_W + RN >= W;
}

// One source row of the gather for the thread's 4 x GBY destinations
// (X0..X0+3, Y0..Y0+GBY-1).  Bit d of DM says whether the row is within
// [-RN, RN+1] rows of destination row d (with GBY = 2 only the first and the
// last source row of the thread's window miss one).  Source column j of the
// strip window is x0-TP+4tx+j; its offset from destination column i is
// kx = j - TP - i, kept in [-RN, RN+1] at compile time.  fy[d] = float(Y0+d)
// in the source row's frame (shifted by H when the row wraps), fxs[i] =
// float(X0+i).  Sources are streamed one float4 chunk (4 columns) at a time.
// CHECK adds the wrap-pass predicate for threads whose source columns wrap the
// torus.
// JA..JB (compile time, inside the window's JLO..JHI) restrict the row to a
// column range, and SHIFTED moves the destinations by xs (a multiple of W) into
// the frame of wrapped sources: an edge thread's passes over exactly the
// chunks that hold their columns, without per-column pass tests.
template <bool WIDE, int RN, bool POW2, bool CHECK, int DM, int GBY, int JA = TP - RN, int JB = TP + 3 + RN + 1,
          bool SHIFTED = false>
__device__ __forceinline__ void gather_row(const float* __restrict__ rxmin, const float* __restrict__ rxmax,
                                           const float* __restrict__ rymin, const float* __restrict__ rymax,
                                           const float* __restrict__ rm, const float (&fy)[GBY + 1],
                                           const float (&fxs)[5], int X0, int gx_base, int W, int cp,
                                           float total_area, float (&acc)[GBY][4], float xs = 0.f) {
    constexpr int JLO = JA, JHI = JB;
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
            float fx0 = 0.f;
            if (CHECK) {
                const int gx = gx_base + j;
                if (wrap_pass(gx, W) != cp) continue;
                fx0 = float(X0 + (gx < 0 ? W : (gx >= W ? -W : 0)));
            }
            const float m = mm[jj];
            float oh[GBY];
#pragma unroll
            for (int d = 0; d < GBY; ++d) {
                if (!((DM >> d) & 1)) continue;
                oh[d] = cell_overlap<WIDE>(fy[d], fy[d + 1], ya[jj], yb[jj]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (j - TP - i < -RN || j - TP - i > RN + 1) continue;
                // exact: integers below 2^24
                const float cx0 = CHECK ? fx0 + float(i) : (SHIFTED ? fxs[i] + xs : fxs[i]);
                const float cx1 = CHECK ? fx0 + float(i + 1) : (SHIFTED ? fxs[i + 1] + xs : fxs[i + 1]);
                const float ow = cell_overlap<WIDE>(cx0, cx1, xa[jj], xb[jj]);
#pragma unroll
                for (int d = 0; d < GBY; ++d) {
                    if (!((DM >> d) & 1)) continue;
                    const float area = __fmul_rn(ow, oh[d]);
                    if (POW2) {
                        // m holds mass * (1 / total_area), exact for a power-of-two
                        // area; a zero area adds a signed zero, which leaves acc
                        // (never -0: it starts at +0) unchanged, so this runs
                        // branch-free.
                        acc[d][i] = __fadd_rn(acc[d][i], __fmul_rn(m, area));
                    } else if (m != 0.f && area > 0.f) {
                        // the division path keeps the reference's skips
                        acc[d][i] = __fadd_rn(acc[d][i], __fmul_rn(m, __fdiv_rn(area, total_area)));
                    }
                }
            }
        }
    }
}

// Terms of the source columns JA..JB of one source row (inside one float4
// chunk), for an x-edge warp: each term is kept in vals and also added to acc
// where `add` holds, so that a lane can take the columns either before or
// after the others.  sh moves the destinations into the frame of wrapped
// sources (a multiple of W, or 0).
template <bool WIDE, int RN, bool POW2, int DM, int GBY, int JA, int JB>
__device__ __forceinline__ void gather_terms(const float* __restrict__ rxmin, const float* __restrict__ rxmax,
                                             const float* __restrict__ rymin, const float* __restrict__ rymax,
                                             const float* __restrict__ rm, const float (&fy)[GBY + 1],
                                             const float (&fxs)[5], float sh, bool add, float total_area,
                                             float (&acc)[GBY][4], float (&vals)[GBY][4][JB - JA + 1]) {
    constexpr int q = JA / 4;
    static_assert(JB / 4 == q, "one chunk of 4 source columns");
    const float4 vxa = *reinterpret_cast<const float4*>(rxmin + 4 * q);
    const float4 vxb = *reinterpret_cast<const float4*>(rxmax + 4 * q);
    const float4 vya = *reinterpret_cast<const float4*>(rymin + 4 * q);
    const float4 vyb = *reinterpret_cast<const float4*>(rymax + 4 * q);
    const float4 vm = *reinterpret_cast<const float4*>(rm + 4 * q);
    const float xa[4] = {vxa.x, vxa.y, vxa.z, vxa.w}, xb[4] = {vxb.x, vxb.y, vxb.z, vxb.w};
    const float ya[4] = {vya.x, vya.y, vya.z, vya.w}, yb[4] = {vyb.x, vyb.y, vyb.z, vyb.w};
    const float mm[4] = {vm.x, vm.y, vm.z, vm.w};
#pragma unroll
    for (int j = JA; j <= JB; ++j) {
        const int jj = j - 4 * q;
        const float m = mm[jj];
        float oh[GBY];
#pragma unroll
        for (int d = 0; d < GBY; ++d) {
            if (!((DM >> d) & 1)) continue;
            oh[d] = cell_overlap<WIDE>(fy[d], fy[d + 1], ya[jj], yb[jj]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (j - TP - i < -RN || j - TP - i > RN + 1) continue;
            const float ow = cell_overlap<WIDE>(__fadd_rn(fxs[i], sh), __fadd_rn(fxs[i + 1], sh), xa[jj], xb[jj]);
#pragma unroll
            for (int d = 0; d < GBY; ++d) {
                if (!((DM >> d) & 1)) continue;
                const float area = __fmul_rn(ow, oh[d]);
                // a term without mass or overlap is +0 or -0, which leaves acc
                // (never -0: it starts at +0) unchanged
                const float v = POW2 ? __fmul_rn(m, area)
                                     : ((m != 0.f && area > 0.f) ? __fmul_rn(m, __fdiv_rn(area, total_area)) : 0.f);
                vals[d][i][j - JA] = v;
                if (add) acc[d][i] = __fadd_rn(acc[d][i], v);
            }
        }
    }
}

// Adds the kept terms of source columns JA..JB where `add` holds, in column order.
template <int RN, int DM, int GBY, int JA, int JB>
__device__ __forceinline__ void gather_add_terms(bool add, float (&acc)[GBY][4],
                                                 const float (&vals)[GBY][4][JB - JA + 1]) {
#pragma unroll
    for (int j = JA; j <= JB; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (j - TP - i < -RN || j - TP - i > RN + 1) continue;
#pragma unroll
            for (int d = 0; d < GBY; ++d) {
                if (!((DM >> d) & 1)) continue;
                if (add) acc[d][i] = __fadd_rn(acc[d][i], vals[d][i][j - JA]);
            }
        }
}

// The 4 x GBY destinations of a thread whose whole source window lies inside
// the torus (no row or column wraps), in a warp whose lanes all do: source
// rows in natural order, one column pass each.  Out of line, so that the
// common case gets its own register allocation and none of the edge paths'
// code.  Taken by the one-row tiles (single world: gather 18.7 -> 18.5 us,
// step 50.8 -> 49.3 us at 512x512); with two rows per thread the call's stack
// frame cost more than it saved (4096-world batch gather 3.40 -> 3.66 ms).
#ifndef FLP_GATHER_INNER_STRIP
#define FLP_GATHER_INNER_STRIP 1
#endif
template <int RN, bool POW2, int GBY, bool WIDE>
__device__ __noinline__ void gather_strip_inner(const float* sxmin, const float* sxmax, const float* symin,
                                                const float* symax, const float* smass, float* __restrict__ out,
                                                int W, int H, float total_area, int x0, int y0, int sw, int tx,
                                                int ty) {
    const int Y0 = y0 + GBY * ty, X0 = x0 + 4 * tx;
    float acc[GBY][4];
#pragma unroll
    for (int d = 0; d < GBY; ++d)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[d][i] = 0.f;
    const int gx_base = x0 - TP + 4 * tx;
    float fxs[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) fxs[i] = float(X0 + i);
    constexpr int NSY = GBY + 2 * RN + 1;
    auto row = [&](auto dm, int r) {
        constexpr int DM = decltype(dm)::value;
        float fy[GBY + 1];
#pragma unroll
        for (int d = 0; d <= GBY; ++d) fy[d] = float(Y0 + d);
        const int off = (GBY * ty + r) * sw + 4 * tx;
        gather_row<WIDE, RN, POW2, false, DM, GBY>(sxmin + off, sxmax + off, symin + off, symax + off, smass + off,
                                                   fy, fxs, X0, gx_base, W, 1, total_area, acc);
    };
    if constexpr (GBY == 1) {
#pragma unroll 1
        for (int r = 0; r < NSY; ++r) row(std::integral_constant<int, 1>(), r);
    } else {
        row(std::integral_constant<int, 1>(), 0);
#pragma unroll 1
        for (int r = 1; r < NSY - 1; ++r) row(std::integral_constant<int, 3>(), r);
        row(std::integral_constant<int, 2>(), NSY - 1);
    }
#pragma unroll
    for (int d = 0; d < GBY; ++d) {
        float* o = out + size_t(Y0 + d) * W;
        if ((W & 3) == 0) {
            *reinterpret_cast<float4*>(o + X0) = make_float4(acc[d][0], acc[d][1], acc[d][2], acc[d][3]);
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) o[X0 + i] = acc[d][i];
        }
    }
}

// Whether one-row tiles (GBY = 1) also take the x-edge path of gather_strip.
#ifndef FLP_GATHER_EDGE_ONE_ROW
#define FLP_GATHER_EDGE_ONE_ROW 0
#endif

// The 4 x GBY destinations of one thread.  Each destination sums its sources
// in the reference's deposit order: row-major over wrapped source indices,
// i.e. rows in wrap-pass order (rows past the bottom edge wrap to the top and
// come first, rows above the top edge come last), then columns the same way.
template <int RN, bool POW2, int GBY, bool WIDE>
__device__ __forceinline__ void gather_strip(const float* sxmin, const float* sxmax, const float* symin,
                                             const float* symax, const float* smass, float* __restrict__ out, int W,
                                             int H, const FlowParams& fp, int x0, int y0, int sw, int tx, int ty) {
    const int Y0 = y0 + GBY * ty, X0 = x0 + 4 * tx;
    float acc[GBY][4];
#pragma unroll
    for (int d = 0; d < GBY; ++d)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[d][i] = 0.f;
    // wrap passes of this thread's window (sources X0-RN .. X0+4+RN, Y0-RN .. Y0+GBY+RN)
    const int rp_lo = (Y0 + GBY + RN >= H) ? 0 : 1, rp_hi = (Y0 - RN < 0) ? 2 : 1;
    const int cp_lo = (X0 + 4 + RN >= W) ? 0 : 1, cp_hi = (X0 - RN < 0) ? 2 : 1;
    const bool xin = cp_lo == 1 && cp_hi == 1;
    // A window that wraps at one side only, with X0 a multiple of 4 and RN <= 3:
    // at the left edge X0 = 0 (sources j < TP wrap), at the right edge of a width
    // divisible by 4 X0 = W - 4 (sources j >= 2 TP wrap); other windows take the
    // generic passes.
    static_assert(RN <= 3 && TP == 4, "edge column ranges assume RN <= 3 and 4-column chunks");
    const bool xleft = cp_hi == 2 && cp_lo == 1 && X0 == 0;
    const bool xright = cp_lo == 0 && cp_hi == 1 && X0 == W - 4 && (W & 3) == 0;
    // Warps that hold an x-edge lane (X0 = 0 or X0 = W - 4) take one path for
    // all their lanes when RN <= 1 and GBY = 2 (with one destination row per
    // thread it made no measurable difference on the 512x512 single world, so
    // it is a compile-time option there): the source columns left of the thread's
    // block (j < TP) and right of it (j >= 2 TP) are computed once, kept in
    // registers and added where each lane's wrapped order puts them (a left
    // edge lane adds the left columns last, a right edge lane the right columns
    // first), instead of the edge and the inside lanes running their passes
    // one after the other.
    bool xedge = false;
    if constexpr (RN <= 1 && (GBY == 2 || FLP_GATHER_EDGE_ONE_ROW)) {
        const bool simple = xin || xleft || xright;
        xedge = __any_sync(__activemask(), xleft || xright) && simple;
    }
    const float shL = xleft ? float(W) : 0.f, shR = xright ? -float(W) : 0.f;
    const int gx_base = x0 - TP + 4 * tx;
    float fxs[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) fxs[i] = float(X0 + i);
    constexpr int NSY = GBY + 2 * RN + 1;  // source rows of the thread's window
    // source row r (global row Y0 - RN + r) in pass rp, for the destination rows DM
    auto row = [&](auto dm, int r, int rp) {
        constexpr int DM = decltype(dm)::value;
        const int gy = Y0 - RN + r;
        if (wrap_pass(gy, H) != rp) return;
        const int yb = Y0 + (gy < 0 ? H : (gy >= H ? -H : 0));
        float fy[GBY + 1];
#pragma unroll
        for (int d = 0; d <= GBY; ++d) fy[d] = float(yb + d);
        const int off = (GBY * ty + r) * sw + 4 * tx;
        if constexpr (RN <= 1 && (GBY == 2 || FLP_GATHER_EDGE_ONE_ROW)) {
            if (xedge) {
                constexpr int RA = 2 * TP, RB = TP + 3 + RN + 1;  // right columns
                float vr[GBY][4][RB - RA + 1];
                gather_terms<WIDE, RN, POW2, DM, GBY, RA, RB>(sxmin + off, sxmax + off, symin + off, symax + off,
                                                              smass + off, fy, fxs, shR, xright, fp.total_area, acc,
                                                              vr);
                if constexpr (RN > 0) {
                    constexpr int LA = TP - RN, LB = TP - 1;  // left columns
                    float vl[GBY][4][LB - LA + 1];
                    gather_terms<WIDE, RN, POW2, DM, GBY, LA, LB>(sxmin + off, sxmax + off, symin + off,
                                                                  symax + off, smass + off, fy, fxs, shL, !xleft,
                                                                  fp.total_area, acc, vl);
                    gather_row<WIDE, RN, POW2, false, DM, GBY, TP, 2 * TP - 1>(
                        sxmin + off, sxmax + off, symin + off, symax + off, smass + off, fy, fxs, X0, gx_base, W, 1,
                        fp.total_area, acc);
                    gather_add_terms<RN, DM, GBY, RA, RB>(!xright, acc, vr);
                    gather_add_terms<RN, DM, GBY, LA, LB>(xleft, acc, vl);
                } else {
                    gather_row<WIDE, RN, POW2, false, DM, GBY, TP, 2 * TP - 1>(
                        sxmin + off, sxmax + off, symin + off, symax + off, smass + off, fy, fxs, X0, gx_base, W, 1,
                        fp.total_area, acc);
                    gather_add_terms<RN, DM, GBY, RA, RB>(!xright, acc, vr);
                }
                return;
            }
        }
        if (xin) {
            gather_row<WIDE, RN, POW2, false, DM, GBY>(sxmin + off, sxmax + off, symin + off, symax + off,
                                                       smass + off, fy, fxs, X0, gx_base, W, 1, fp.total_area, acc);
        } else if (xleft) {
            // X0 = 0: columns j >= TP are inside, j < TP wrap to the right edge and come last
            gather_row<WIDE, RN, POW2, false, DM, GBY, TP, TP + 3 + RN + 1>(
                sxmin + off, sxmax + off, symin + off, symax + off, smass + off, fy, fxs, X0, gx_base, W, 1,
                fp.total_area, acc);
            gather_row<WIDE, RN, POW2, false, DM, GBY, TP - RN, TP - 1, true>(
                sxmin + off, sxmax + off, symin + off, symax + off, smass + off, fy, fxs, X0, gx_base, W, 2,
                fp.total_area, acc, float(W));
        } else if (xright) {
            // X0 = W - 4: columns j >= 2 TP wrap to the left edge and come first, j < 2 TP are inside
            gather_row<WIDE, RN, POW2, false, DM, GBY, 2 * TP, TP + 3 + RN + 1, true>(
                sxmin + off, sxmax + off, symin + off, symax + off, smass + off, fy, fxs, X0, gx_base, W, 0,
                fp.total_area, acc, -float(W));
            gather_row<WIDE, RN, POW2, false, DM, GBY, TP - RN, 2 * TP - 1>(
                sxmin + off, sxmax + off, symin + off, symax + off, smass + off, fy, fxs, X0, gx_base, W, 1,
                fp.total_area, acc);
        } else {
            for (int cp = cp_lo; cp <= cp_hi; ++cp)
                gather_row<WIDE, RN, POW2, true, DM, GBY>(sxmin + off, sxmax + off, symin + off, symax + off,
                                                          smass + off, fy, fxs, X0, gx_base, W, cp, fp.total_area,
                                                          acc);
        }
    };
    for (int rp = rp_lo; rp <= rp_hi; ++rp) {
        if constexpr (GBY == 1) {
#pragma unroll 1
            for (int r = 0; r < NSY; ++r) row(std::integral_constant<int, 1>(), r, rp);
        } else {
            static_assert(GBY == 2, "row masks are written out for one or two destination rows per thread");
            // the first source row reaches destination row 0 only, the last row 1 only
            row(std::integral_constant<int, 1>(), 0, rp);
#pragma unroll 1
            for (int r = 1; r < NSY - 1; ++r) row(std::integral_constant<int, 3>(), r, rp);
            row(std::integral_constant<int, 2>(), NSY - 1, rp);
        }
    }
#pragma unroll
    for (int d = 0; d < GBY; ++d) {
        if (Y0 + d >= H) break;
        float* o = out + size_t(Y0 + d) * W;
        if (X0 + 3 < W && (W & 3) == 0) {
            *reinterpret_cast<float4*>(o + X0) = make_float4(acc[d][0], acc[d][1], acc[d][2], acc[d][3]);
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (X0 + i < W) o[X0 + i] = acc[d][i];
        }
    }
}

// Thread (tx, ty) of a gather tile.  Tiles inside the torus map a warp to
// 16 x 2 threads.  Tiles whose sources reach across an x edge use a
// column-major mapping (a warp is 2 x 16 threads), which puts the threads that
// need more than one column pass into the two edge warps; its lane order
// keeps the rows read by a quarter-warp in distinct bank groups of the
// 76-float rows (GBY = 1: 8 consecutive thread rows of one column; GBY = 2:
// 4 thread rows of two columns).
//
// For GBY = 2 the x-edge tiles take a lane table (tx | ty << 4 per thread):
// warp 0 holds the two edge columns tx = 0 and 15 (it takes the x-edge path
// of gather_strip), warp 1 the top and bottom thread rows ty = 0 and 15 of the
// inner columns (the lanes whose source rows wrap in a tile on a y edge, so
// that only two warps run a second row pass), the other six warps the inner
// block.  Every quarter-warp of the table reads distinct 16-byte bank groups
// of the 76-float rows ((6 ty + tx) mod 8 all different).
static __device__ const unsigned char kGatherEdgeLanes2[256] = {
      0,  15,  16,  31,  32,  47,  48,  63,  64,  79,  80,  95,  96, 111, 112, 127,
    128, 143, 144, 159, 160, 175, 176, 191, 192, 207, 208, 223, 224, 239, 240, 255,
     10, 251, 241,   6,   4, 254,   7,   9,  11,  20,  14,  13, 250,   8,   1, 253,
      2, 249, 243,  26, 252,  25, 247,  12, 248,   3,  19, 246,   5, 244, 245, 242,
    148,  57,  52,  33, 210,  58,  35, 137, 139, 220,  70, 217,  41, 204, 146, 173,
     46, 140, 227, 116, 197, 113,  62,  37, 102,  98, 205,  30,  61, 177,  65, 190,
    215, 130,  42,  40,  53, 213, 155, 218,  69,  38,  86, 206,  67, 201, 136, 107,
    169,  68, 170, 110, 195,  81,  90,  83,  23,  60, 232, 221,  92, 209, 236, 219,
    150, 124, 131,  56, 133, 172,  71, 237, 226, 120, 214, 164, 231, 171, 115, 109,
    162, 202,  76,  72, 185, 125, 187, 193, 238, 216, 104, 100,  93, 189, 123, 129,
    158,  78,  18,  66,  89,  77, 119,  29,  54, 188,  22, 153,  97, 156, 101, 103,
     44, 180,  43, 184, 222,  73, 161,  75, 126, 142, 235, 122,  45, 138, 203, 141,
     36, 117,  34,  91, 178, 166, 167, 105, 199, 228, 168, 234,  74, 183, 121, 233,
    181, 108, 106,  50, 230, 149, 229, 179, 135, 118, 196,  88,  85, 174,  27, 225,
    154, 212, 145,  21,  24, 114,  51, 147, 200,  84,  87,  99, 198,  49, 132, 211,
    182, 194, 151,  17, 134, 157, 165,  94,  28, 163,  82, 152,  55,  39, 186,  59,
};

template <int GBY>
__device__ __forceinline__ void gather_thread(bool cm, bool table, int& tx, int& ty) {
    const int tid = threadIdx.x;
    if (!cm) {
        tx = tid & 15;
        ty = tid >> 4;
    } else if (GBY == 2 && table) {
        const int v = kGatherEdgeLanes2[tid];
        tx = v & 15;
        ty = v >> 4;
    } else if (GBY == 1) {
        tx = tid >> 4;
        ty = tid & 15;
    } else {
        tx = 2 * (tid >> 5) + (tid & 1);
        ty = (tid & 31) >> 1;
    }
}

// Out of line: each (RN, POW2, GBY) instantiation gets its own register
// allocation instead of sharing the calling kernel's with the wider windows
// (inlined together, the batched gather spilled in its common RN = 1 path).
template <int RN, bool POW2, int GBY, bool WIDE = false>
__device__ __noinline__ void gather_body(float* sm, const float* __restrict__ DX, const float* __restrict__ DY,
                            const float* __restrict__ A, float* __restrict__ out, int W, int H, const FlowParams& fp,
                            int x0, int y0) {
    constexpr int SRH = gt_h(GBY) + 2 * RN + 1;
    const int tid = threadIdx.x;
    const bool cm = gather_column_major(x0, W, RN);
    // the lane table when the tile's x-edge lanes are tx = 0 and tx = 15 only
    const bool table = x0 + GT_W + RN < W || x0 + GT_W == W;
    int tx, ty;
    gather_thread<GBY>(cm, table, tx, ty);
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
    // stage destinations and states (dx -> xmin in place, dy -> ymin in place,
    // state -> source mass in place)
    if (cm) stage_sources<SRH, SR_W>(sxmin, symin, smass, DX, DY, A, colx, rowy, W);
    else stage_sources<SRH, SR_W - 4>(sxmin, symin, smass, DX, DY, A, colx, rowy, W);
    cp_async_wait_all();
    __syncthreads();
    for (int i = 4 * tid; i < sw * SRH; i += 1024) {
        const float4 dx = *reinterpret_cast<const float4*>(sxmin + i);
        const float4 dy = *reinterpret_cast<const float4*>(symin + i);
        const float4 a = *reinterpret_cast<const float4*>(smass + i);
        *reinterpret_cast<float4*>(smass + i) = make_float4(source_mass<POW2>(a.x, fp), source_mass<POW2>(a.y, fp),
                                                            source_mass<POW2>(a.z, fp), source_mass<POW2>(a.w, fp));
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
    if (y0 + GBY * ty < H && x0 + 4 * tx < W)
    {
        const int Y0 = y0 + GBY * ty, X0 = x0 + 4 * tx;
        // a lane whose window wraps neither a row nor a column of the torus
        const bool inner = Y0 - RN >= 0 && Y0 + GBY + RN < H && X0 - RN >= 0 && X0 + 4 + RN < W;
        if (FLP_GATHER_INNER_STRIP && GBY == 1 && __all_sync(__activemask(), inner))
            gather_strip_inner<RN, POW2, GBY, WIDE>(sxmin, sxmax, symin, symax, smass, out, W, H, fp.total_area, x0,
                                                    y0, sw, tx, ty);
        else
            gather_strip<RN, POW2, GBY, WIDE>(sxmin, sxmax, symin, symax, smass, out, W, H, fp, x0, y0, sw, tx, ty);
    }
    __syncthreads();
}

// Reintegrated mass at destination (X, Y) for any window, sources read from
// the destination and state planes in global memory.  Handles the
// nearest-cell mode, the reference's [-W, 2W] cell clamp, and windows wider
// than the grid.
template <bool POW2, class T>
__device__ T gather_generic_2d(const T* __restrict__ DX, const T* __restrict__ DY, const T* __restrict__ A, int W,
                               int H, int X, int Y, int R, const FlowParams& fp) {
    const T s = T(fp.s);
    T acc = T(0);
    for (int jy = 0; jy <= 2 * R; ++jy) {
        const int ky = rotated_offset(jy, Y, R, H);
        const int yw = wrap_coord(Y + ky, H);
        const int iy = yw - ky;
        for (int jx = 0; jx <= 2 * R; ++jx) {
            const int kx = rotated_offset(jx, X, R, W);
            const int xw = wrap_coord(X + kx, W);
            const int ix = xw - kx;
            const size_t src = size_t(yw) * W + xw;
            const T m = source_mass<POW2>(A[src], fp);
            if (m == T(0)) continue;
            const T dx = DX[src], dy = DY[src];
            if (fp.point_mode) {
                if (f2i_sat(round(dx)) == ix && f2i_sat(round(dy)) == iy) acc = rn_add(acc, m);
                continue;
            }
            const T xmin = rn_sub(dx, s), xmax = rn_add(dx, s);
            const T ymin = rn_sub(dy, s), ymax = rn_add(dy, s);
            const int ix_lo = max(f2i_sat(floor(xmin)), -W), ix_hi = min(f2i_sat(ceil(xmax)), 2 * W);
            const int iy_lo = max(f2i_sat(floor(ymin)), -H), iy_hi = min(f2i_sat(ceil(ymax)), 2 * H);
            if (ix < ix_lo || ix > ix_hi || iy < iy_lo || iy > iy_hi) continue;
            const T ox0 = fmax(T(ix), xmin), ox1 = fmin(T(ix + 1), xmax);
            const T oy0 = fmax(T(iy), ymin), oy1 = fmin(T(iy + 1), ymax);
            const T ow = fmax(rn_sub(ox1, ox0), T(0));
            const T oh = fmax(rn_sub(oy1, oy0), T(0));
            const T area = rn_mul(ow, oh);
            if (!(area > T(0))) continue;
            acc = rn_add(acc, POW2 ? rn_mul(m, area) : rn_mul(m, rn_div(area, T(fp.total_area))));
        }
    }
    return acc;
}

// One 64 x (16 * GBY) tile of one channel of gather_2d; `sm` holds
// gather_smem_bytes_inl(GBY).  dxc/dyc are that channel's destination planes,
// ac its state plane (the sources' masses), out its next-state plane.
template <bool POW2, int GBY>
__device__ void gather_item(float* sm, const float* __restrict__ dxc, const float* __restrict__ dyc,
                            const float* __restrict__ ac, float* __restrict__ out, int W, int H,
                            const FlowParams& fp, int dmax_bits, int x0, int y0) {
    const int RN = window_from_dmax(dmax_bits, fp, max(W, H));
    const bool fast = RN <= RN_MAX && 2 * RN + 2 <= W && 2 * RN + 2 <= H && !fp.point_mode;
    if (fast) {
        // the saturating overlap form pays where each x overlap serves two
        // destination rows; with one row the min/max form measured faster
        // (512x512 single world 19.1 vs 20.3 us)
        if (POW2 && GBY == 2 && fp.wide_square) {
            switch (RN) {
                case 0: gather_body<0, true, GBY, true>(sm, dxc, dyc, ac, out, W, H, fp, x0, y0); break;
                case 1: gather_body<1, true, GBY, true>(sm, dxc, dyc, ac, out, W, H, fp, x0, y0); break;
                case 2: gather_body<2, true, GBY, true>(sm, dxc, dyc, ac, out, W, H, fp, x0, y0); break;
                default: gather_body<3, true, GBY, true>(sm, dxc, dyc, ac, out, W, H, fp, x0, y0); break;
            }
            return;
        }
        switch (RN) {
            case 0: gather_body<0, POW2, GBY>(sm, dxc, dyc, ac, out, W, H, fp, x0, y0); break;
            case 1: gather_body<1, POW2, GBY>(sm, dxc, dyc, ac, out, W, H, fp, x0, y0); break;
            case 2: gather_body<2, POW2, GBY>(sm, dxc, dyc, ac, out, W, H, fp, x0, y0); break;
            default: gather_body<3, POW2, GBY>(sm, dxc, dyc, ac, out, W, H, fp, x0, y0); break;
        }
        return;
    }
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll 1
    for (int d = 0; d < GBY; ++d) {
        const int Y = y0 + GBY * ty + d;
#pragma unroll 1
        for (int i = 0; i < 4; ++i) {
            const int X = x0 + 4 * tx + i;
            if (X < W && Y < H)
                out[size_t(Y) * W + X] = gather_generic_2d<POW2>(dxc, dyc, ac, W, H, X, Y, RN + 1, fp);
        }
    }
}

}  // namespace flp
