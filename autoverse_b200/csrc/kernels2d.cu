// 2D step kernels of the Flow Lenia engine (sm_100a):
//   * conv_direct_growth_2d — shared-memory tiled torus convolution with the
//     growth function and the per-target weighted sum fused into its epilogue
//     (src/compute/fft.rs:288-324 + growth.rs:45-59 + propagator.rs:270-279);
//   * transport_2d — one pass that forms the channel sum, both Sobel
//     gradients, alpha, the flow and the reintegrated mass, in gather form
//     (propagator.rs:304-371, gradient.rs:68-108, flow.rs:68-87,
//     reintegration.rs:60-167);
//   * the flow-bound reduction and the FP64 compensated mass reduction.
//
// Arithmetic that the reference performs in f32 is written with explicit
// round-to-nearest intrinsics (__fadd_rn/__fmul_rn/...) so that nvcc cannot
// contract it into FMAs: the per-source destinations, overlap areas and
// deposited masses are then bit-identical to the reference's, and the gather
// visits sources in the reference's scatter order, so the transport stage
// reproduces CpuPropagator bit for bit given the same affinity field.
#include "common.cuh"
#include "kernels.h"

#include <math.h>

namespace flp {

// ---------------------------------------------------------------------------
// Direct convolution + growth.
// Block 32x8 threads, tile 32x32 outputs (4 per thread, rows ty+8i).
// blockIdx.z selects the target channel; kernels targeting it are applied in
// kernel order and their weighted growth is accumulated in that order.
// ---------------------------------------------------------------------------
constexpr int CD_TW = 32, CD_TH = 32;

__global__ void __launch_bounds__(256) conv_direct_growth_2d(const float* __restrict__ A, float* __restrict__ U,
                                                             const KDesc* __restrict__ kd, int K,
                                                             const float* __restrict__ taps, int W, int H, int rmax,
                                                             int* reset_slot, int nreset) {
    extern __shared__ float sm[];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * 32 + tx;
    const int c = blockIdx.z;
    const int x0 = blockIdx.x * CD_TW, y0 = blockIdx.y * CD_TH;
    const size_t N = size_t(W) * H;
    if (reset_slot && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && tid == 0)
        reset_bound_slots(reset_slot, nreset);
    const int Pmax = CD_TW + 2 * rmax;
    float* tile = sm;                                   // (CD_TH + 2r) x (CD_TW + 2r)
    float* tsm = sm + size_t(CD_TH + 2 * rmax) * Pmax;  // taps
    float accu[4] = {0.f, 0.f, 0.f, 0.f};
    int loaded_src = -1, loaded_r = -1;
    for (int k = 0; k < K; ++k) {
        const KDesc d = kd[k];
        if (d.tgt != c) continue;
        const int r = d.r, side = 2 * r + 1, P = CD_TW + 2 * r;
        __syncthreads();
        for (int i = tid; i < side * side; i += 256) tsm[i] = taps[d.tap_off + i];
        if (d.src != loaded_src || r != loaded_r) {
            const float* a = A + size_t(d.src) * N;
            const int rows = CD_TH + 2 * r;
            for (int i = tid; i < rows * P; i += 256) {
                int ly = i / P, lx = i - ly * P;
                int gy = wrap_coord(y0 - r + ly, H), gx = wrap_coord(x0 - r + lx, W);
                tile[i] = a[size_t(gy) * W + gx];
            }
            loaded_src = d.src;
            loaded_r = r;
        }
        __syncthreads();
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int dy = 0; dy < side; ++dy) {
            const float* trow = tsm + dy * side;
            const float* base = tile + (ty + dy) * P + tx;
            for (int dx = 0; dx < side; ++dx) {
                const float t = trow[dx];
#pragma unroll
                for (int i = 0; i < 4; ++i) acc[i] = fmaf(t, base[(8 * i) * P + dx], acc[i]);
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float diff = __fsub_rn(acc[i], d.mu);
            float e = expf(__fmul_rn(__fmul_rn(-diff, diff), d.inv2s2));
            float g = __fsub_rn(__fmul_rn(2.0f, e), 1.0f);
            accu[i] = __fadd_rn(accu[i], __fmul_rn(d.weight, g));
        }
    }
    float* u = U + size_t(c) * N;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int y = y0 + ty + 8 * i, x = x0 + tx;
        if (x < W && y < H) u[size_t(y) * W + x] = accu[i];
    }
}

size_t conv_direct_smem_bytes(int rmax) {
    int P = CD_TW + 2 * rmax;
    int side = 2 * rmax + 1;
    return sizeof(float) * (size_t(CD_TH + 2 * rmax) * P + size_t(side) * side);
}

void launch_conv_direct_2d(const float* A, float* U, const KDesc* kd, int K, const float* taps, int W, int H, int C,
                           int rmax, int* reset_slot, cudaStream_t st) {
    dim3 grid((W + CD_TW - 1) / CD_TW, (H + CD_TH - 1) / CD_TH, C);
    size_t smem = conv_direct_smem_bytes(rmax);
    conv_direct_growth_2d<<<grid, dim3(32, 8), smem, st>>>(A, U, kd, K, taps, W, H, rmax, reset_slot, C);
}

// ---------------------------------------------------------------------------
// Gather window from the flow bound.
// |F_x|,|F_y| <= max(max|grad U|, max|grad A_sum|) since F = (1-a)gU - a gA
// with a in [0,1]; the Sobel/8 of a field ranges over at most half its spread,
// |U| <= sum_k |w_k| (G in [-1,1]) and the spread of A_sum is at most
// sum_c (max A_c - min A_c).  With |dest - x| <= D, a source at x overlaps
// cell ix only if x - ix lies in (-(D+s), D+s+1) (reintegration.rs:105-146),
// so sources x = ix + k with k in [-RN, RN+1], RN = ceil(D+s) - 1, cover every
// deposit.  D carries a margin for the rounding of dest and x_min/x_max.
// bound: C pairs (max, min) as ordered ints.  Returns RN.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int gather_window(const int* bound, int C, const FlowParams& fp, int maxside, int* status) {
    float hi = 0.f, lo = 0.f;
    for (int c = 0; c < C; ++c) {
        hi += ordered_to_float(bound[2 * c]);
        lo += ordered_to_float(bound[2 * c + 1]);
    }
    float spread = (hi - lo) * 1.0001f;
    if (!(spread >= 0.f) || !isfinite(spread)) {
        if (status && threadIdx.x == 0 && threadIdx.y == 0) atomicOr(status, STATUS_NONFINITE);
        return 0;
    }
    float fb = fmaxf(fp.ubound, 0.5f * spread);
    float Db = fp.dt * fb * 1.0001f + fp.pos_eps;
    float rn = ceilf(Db + fp.s) - 1.0f;
    int cap = 2 * maxside + 2;
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

// Overlap contribution of one source square (x_min..x_max, y_min..y_max) to
// cell (ix, iy): reintegration.rs:129-157, in the reference's order.
__device__ __forceinline__ float overlap_mass(float mass, float xmin, float xmax, float ymin, float ymax, int ix, int iy,
                                              const FlowParams& fp) {
    float ox0 = fmaxf(float(ix), xmin), ox1 = fminf(float(ix + 1), xmax);
    float oy0 = fmaxf(float(iy), ymin), oy1 = fminf(float(iy + 1), ymax);
    float ow = fmaxf(__fsub_rn(ox1, ox0), 0.f);
    float oh = fmaxf(__fsub_rn(oy1, oy0), 0.f);
    float area = __fmul_rn(ow, oh);
    if (!(area > 0.f)) return 0.f;
    float frac = fp.area_pow2 ? __fmul_rn(area, fp.inv_area) : __fdiv_rn(area, fp.total_area);
    return __fmul_rn(mass, frac);
}

__device__ __forceinline__ int f2i_sat(float v) {
    // Rust `f32 as i32`: saturating, NaN -> 0.
    if (v != v) return 0;
    if (v >= 2147483647.f) return 2147483647;
    if (v <= -2147483648.f) return -2147483647 - 1;
    return int(v);
}

// Flow at a wrapped source cell, read straight from global memory.
__device__ void source_dest_global(const float* __restrict__ A, const float* __restrict__ Uc, int C, int W, int H,
                                   int xw, int yw, const FlowParams& fp, float& dest_x, float& dest_y) {
    const size_t N = size_t(W) * H;
    int xs[3] = {wrap_coord(xw - 1, W), xw, wrap_coord(xw + 1, W)};
    int ys[3] = {wrap_coord(yw - 1, H), yw, wrap_coord(yw + 1, H)};
    float as[3][3], us[3][3];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            size_t idx = size_t(ys[j]) * W + xs[i];
            float s = 0.f;
            for (int c = 0; c < C; ++c) s = __fadd_rn(s, A[size_t(c) * N + idx]);
            as[j][i] = s;
            us[j][i] = Uc[idx];
        }
    float gax, gay, gux, guy;
    sobel2(as[0][0], as[0][1], as[0][2], as[1][0], as[1][2], as[2][0], as[2][1], as[2][2], gax, gay);
    sobel2(us[0][0], us[0][1], us[0][2], us[1][0], us[1][2], us[2][0], us[2][1], us[2][2], gux, guy);
    float alpha = flow_alpha(as[1][1], fp.beta_a, fp.nexp);
    float oma = __fsub_rn(1.0f, alpha);
    float fx = __fsub_rn(__fmul_rn(oma, gux), __fmul_rn(alpha, gax));
    float fy = __fsub_rn(__fmul_rn(oma, guy), __fmul_rn(alpha, gay));
    dest_x = __fadd_rn(float(xw), __fmul_rn(fp.dt, fx));
    dest_y = __fadd_rn(float(yw), __fmul_rn(fp.dt, fy));
}

// Reintegrated mass of channel c at destination (X, Y), any radius, sources
// evaluated from global memory.  Handles the nearest-cell mode, the
// reference's [-W, 2W] cell clamp, and radii wider than the grid.
__device__ float gather_generic_2d(const float* __restrict__ A, const float* __restrict__ U, int c, int C, int W, int H,
                                   int X, int Y, int R, const FlowParams& fp) {
    const size_t N = size_t(W) * H;
    const float* Ac = A + size_t(c) * N;
    const float* Uc = U + size_t(c) * N;
    float acc = 0.f;
    for (int jy = 0; jy <= 2 * R; ++jy) {
        int ky = rotated_offset(jy, Y, R, H);
        int yw = wrap_coord(Y + ky, H);
        int iy = yw - ky;
        for (int jx = 0; jx <= 2 * R; ++jx) {
            int kx = rotated_offset(jx, X, R, W);
            int xw = wrap_coord(X + kx, W);
            int ix = xw - kx;
            float mass = Ac[size_t(yw) * W + xw];
            if (fabsf(mass) < 1e-10f) continue;
            float dx, dy;
            source_dest_global(A, Uc, C, W, H, xw, yw, fp, dx, dy);
            if (fp.point_mode) {
                if (f2i_sat(roundf(dx)) == ix && f2i_sat(roundf(dy)) == iy) acc = __fadd_rn(acc, mass);
                continue;
            }
            float xmin = __fsub_rn(dx, fp.s), xmax = __fadd_rn(dx, fp.s);
            float ymin = __fsub_rn(dy, fp.s), ymax = __fadd_rn(dy, fp.s);
            int ix_lo = max(f2i_sat(floorf(xmin)), -W), ix_hi = min(f2i_sat(ceilf(xmax)), 2 * W);
            int iy_lo = max(f2i_sat(floorf(ymin)), -H), iy_hi = min(f2i_sat(ceilf(ymax)), 2 * H);
            if (ix < ix_lo || ix > ix_hi || iy < iy_lo || iy > iy_hi) continue;
            acc = __fadd_rn(acc, overlap_mass(mass, xmin, xmax, ymin, ymax, ix, iy, fp));
        }
    }
    return acc;
}

// ---------------------------------------------------------------------------
// Fused transport.  Block = (64x16 tile, one channel), 256 threads; thread
// (tx, ty) owns the 4-cell row strip x0+4tx.., y0+ty.  The source region is
// the tile plus R rows above/below and TP(=4) columns left/right (columns
// padded to keep float4 alignment); the Sobel inputs add a 1-cell ring.
// Per source the kernel stores its square's bounds x_min, x_max, y_min, y_max
// (reintegration.rs:105-108) and its mass; destinations then gather.
// ---------------------------------------------------------------------------
#ifndef TRANSPORT_MIN_BLOCKS
#define TRANSPORT_MIN_BLOCKS 2
#endif
// Fused transport.  Block = (64x16 tile, one channel), 256 threads; thread
// (tx, ty) owns the 4-cell row strip x0+4tx.., y0+ty.  Sources are the cells
// y0-RN .. y0+15+RN+1 by x0-TP .. x0+63+TP (columns padded to keep float4
// alignment); the Sobel inputs add a 1-cell ring.  Per source the block
// stores its square's bounds x_min, x_max, y_min, y_max
// (reintegration.rs:105-108) and its mass; destinations then gather.
constexpr int TT_W = 64, TT_H = 16, TP = 4, RN_MAX = 3;
constexpr int SR_W = TT_W + 2 * TP;              // 72 source columns
constexpr int SR_HMAX = TT_H + 2 * RN_MAX + 1;   // up to 23 source rows
constexpr int AR_W = SR_W + 2;                   // 74 with the Sobel ring
constexpr int AR_HMAX = SR_HMAX + 2;             // up to 25
constexpr int SRC_CHUNK = 8;                     // sources per thread in the sliding Sobel

// Region arrays are padded to a multiple of 4 floats so that every array,
// and hence every float4 chunk of the source arrays, is 16-byte aligned.
__host__ __device__ constexpr int region_floats(int arh) { return ((AR_W * arh + 3) / 4) * 4; }
static_assert(SR_W % 4 == 0, "source rows must stay 16-byte aligned");

size_t transport_smem_bytes() { return sizeof(float) * (3 * region_floats(AR_HMAX) + 5 * SR_W * SR_HMAX); }

__device__ __forceinline__ int wrap_pass(int g, int size) { return g >= size ? 0 : (g < 0 ? 2 : 1); }

// Block max/min into an ordered-int slot pair.  A non-finite value anywhere
// in the block publishes +inf as the max, so the next gather_window sees a
// non-finite spread and raises STATUS_NONFINITE.
__device__ __forceinline__ void block_minmax_atomic(float vmax, float vmin, bool bad, int* slot) {
    __shared__ float red_max[32], red_min[32];
    const int anybad = __syncthreads_or(bad ? 1 : 0);
    for (int o = 16; o > 0; o >>= 1) {
        vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
    }
    int tid = threadIdx.y * blockDim.x + threadIdx.x;
    int warp = tid >> 5, lane = tid & 31;
    if (lane == 0) { red_max[warp] = vmax; red_min[warp] = vmin; }
    __syncthreads();
    if (tid == 0) {
        int nw = (blockDim.x * blockDim.y) >> 5;
        float mx = red_max[0], mn = red_min[0];
        for (int w = 1; w < nw; ++w) { mx = fmaxf(mx, red_max[w]); mn = fminf(mn, red_min[w]); }
        if (anybad) mx = INFINITY;
        atomicMax(slot + 0, float_to_ordered(mx));
        atomicMin(slot + 1, float_to_ordered(mn));
    }
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
                                           int W, int cp, float inv_or_total, float (&acc)[4]) {
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
            if (m == 0.f) continue;
            const float oy0 = fmaxf(cy0, ya[jj]), oy1 = fminf(cy1, yb[jj]);
            const float oh = fmaxf(__fsub_rn(oy1, oy0), 0.f);
            if (!(oh > 0.f)) continue;
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
                    acc[i] = __fadd_rn(acc[i], __fmul_rn(m, __fdiv_rn(area, inv_or_total)));
                }
            }
        }
    }
}

template <int RN, bool POW2>
__device__ void transport_body(float* sm, const float* __restrict__ A, const float* __restrict__ U,
                               float* __restrict__ Anext, int c, int C, int W, int H, const FlowParams& fp,
                               float (&out)[4]) {
    constexpr int SRH = TT_H + 2 * RN + 1, ARH = SRH + 2, AREG = region_floats(ARH);
    float* asum = sm;                   // ARH x AR_W: channel sum
    float* usm = asum + AREG;           // ARH x AR_W: U_c
    float* amc = usm + AREG;            // ARH x AR_W: A_c
    float* sxmin = amc + AREG;          // SRH x SR_W each (16-byte aligned)
    float* sxmax = sxmin + SR_W * SRH;
    float* symin = sxmax + SR_W * SRH;
    float* symax = symin + SR_W * SRH;
    float* smass = symax + SR_W * SRH;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int x0 = blockIdx.x * TT_W, y0 = blockIdx.y * TT_H;
    const size_t N = size_t(W) * H;
    const float* Uc = U + size_t(c) * N;
    const float s = fp.s;

    // channel sum, U_c and A_c over the source region plus the Sobel ring
    for (int i = tid; i < AR_W * ARH; i += 256) {
        const int ly = i / AR_W, lx = i - ly * AR_W;
        const int gy = wrap_near(y0 - RN - 1 + ly, H), gx = wrap_near(x0 - TP - 1 + lx, W);
        const size_t idx = size_t(gy) * W + gx;
        float a = 0.f, mine = 0.f;
        for (int k = 0; k < C; ++k) {
            const float v = A[size_t(k) * N + idx];
            a = __fadd_rn(a, v);
            if (k == c) mine = v;
        }
        asum[i] = a;
        amc[i] = mine;
        usm[i] = Uc[idx];
    }
    __syncthreads();
    // Per-source square bounds and (scaled) mass.  Each thread walks a column
    // segment of SRC_CHUNK sources with a 3-row register window of the channel
    // sum and U_c.
    {
        constexpr int COL0 = TP - RN, NCOL = TT_W + 2 * RN + 1;
        constexpr int NCH = (SRH + SRC_CHUNK - 1) / SRC_CHUNK;
        for (int item = tid; item < NCOL * NCH; item += 256) {
            const int col = item % NCOL, ch = item / NCOL;
            const int sx = COL0 + col, r0 = ch * SRC_CHUNK;
            const int xw = wrap_near(x0 - TP + sx, W);
            const float* ap = asum + r0 * AR_W + sx;  // region row r0 = source row r0 - 1
            const float* up = usm + r0 * AR_W + sx;
            float a0[3] = {ap[0], ap[1], ap[2]}, a1[3] = {ap[AR_W], ap[AR_W + 1], ap[AR_W + 2]};
            float u0[3] = {up[0], up[1], up[2]}, u1[3] = {up[AR_W], up[AR_W + 1], up[AR_W + 2]};
#pragma unroll
            for (int r = 0; r < SRC_CHUNK; ++r) {
                const int sy = r0 + r;
                if (sy >= SRH) break;
                const float* ar = ap + (r + 2) * AR_W;
                const float* ur = up + (r + 2) * AR_W;
                const float a2[3] = {ar[0], ar[1], ar[2]};
                const float u2[3] = {ur[0], ur[1], ur[2]};
                const int yw = wrap_near(y0 - RN + sy, H);
                float mass = amc[(sy + 1) * AR_W + sx + 1];
                if (fabsf(mass) < 1e-10f) mass = 0.f;
                float gax, gay, gux, guy;
                sobel2(a0[0], a0[1], a0[2], a1[0], a1[2], a2[0], a2[1], a2[2], gax, gay);
                sobel2(u0[0], u0[1], u0[2], u1[0], u1[2], u2[0], u2[1], u2[2], gux, guy);
                const float alpha = flow_alpha(a1[1], fp.beta_a, fp.nexp);
                const float oma = __fsub_rn(1.0f, alpha);
                const float fx = __fsub_rn(__fmul_rn(oma, gux), __fmul_rn(alpha, gax));
                const float fy = __fsub_rn(__fmul_rn(oma, guy), __fmul_rn(alpha, gay));
                const float dx = __fadd_rn(float(xw), __fmul_rn(fp.dt, fx));
                const float dy = __fadd_rn(float(yw), __fmul_rn(fp.dt, fy));
                const int o = sy * SR_W + sx;
                sxmin[o] = __fsub_rn(dx, s);
                sxmax[o] = __fadd_rn(dx, s);
                symin[o] = __fsub_rn(dy, s);
                symax[o] = __fadd_rn(dy, s);
                smass[o] = POW2 ? __fmul_rn(mass, fp.inv_area) : mass;
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    a0[t] = a1[t]; a1[t] = a2[t];
                    u0[t] = u1[t]; u1[t] = u2[t];
                }
            }
        }
    }
    __syncthreads();

    const int Y = y0 + ty, X0 = x0 + 4 * tx;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    if (Y < H && X0 < W) {
        const int rp_lo = (y0 + TT_H + RN >= H) ? 0 : 1, rp_hi = (y0 - RN < 0) ? 2 : 1;
        const int cp_lo = (x0 + TT_W + RN >= W) ? 0 : 1, cp_hi = (x0 - RN < 0) ? 2 : 1;
        const bool xin = cp_lo == 1 && cp_hi == 1;
        const int gx_base = x0 - TP + 4 * tx;
        const float inv_or_total = POW2 ? fp.inv_area : fp.total_area;
        for (int rp = rp_lo; rp <= rp_hi; ++rp) {
#pragma unroll 1
            for (int ky = -RN; ky <= RN + 1; ++ky) {
                const int gy = Y + ky;
                if (wrap_pass(gy, H) != rp) continue;
                const int iy = Y + (gy < 0 ? H : (gy >= H ? -H : 0));
                const float cy0 = float(iy), cy1 = float(iy + 1);
                const int off = (ty + RN + ky) * SR_W + 4 * tx;
                if (xin) {
                    gather_row<RN, POW2, false>(sxmin + off, sxmax + off, symin + off, symax + off, smass + off,
                                                cy0, cy1, X0, gx_base, W, 1, inv_or_total, acc);
                } else {
                    for (int cp = cp_lo; cp <= cp_hi; ++cp)
                        gather_row<RN, POW2, true>(sxmin + off, sxmax + off, symin + off, symax + off, smass + off,
                                                   cy0, cy1, X0, gx_base, W, cp, inv_or_total, acc);
                }
            }
        }
        float* o = Anext + size_t(c) * N + size_t(Y) * W;
        if (X0 + 3 < W && (W & 3) == 0) {
            *reinterpret_cast<float4*>(o + X0) = make_float4(acc[0], acc[1], acc[2], acc[3]);
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (X0 + i < W) o[X0 + i] = acc[i];
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) out[i] = acc[i];
}

template <bool POW2>
__global__ void __launch_bounds__(256, TRANSPORT_MIN_BLOCKS) transport_2d(const float* __restrict__ A,
                                                                          const float* __restrict__ U,
                                                                          float* __restrict__ Anext, int C, int W,
                                                                          int H, FlowParams fp,
                                                                          const int* __restrict__ bound_in,
                                                                          int* bound_out, int* status) {
    extern __shared__ __align__(16) float sm[];
    const int c = blockIdx.z;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int x0 = blockIdx.x * TT_W, y0 = blockIdx.y * TT_H;
    const size_t N = size_t(W) * H;
    const int RN = gather_window(bound_in, C, fp, max(W, H), status);
    float out[4] = {0.f, 0.f, 0.f, 0.f};
    const bool fast = RN <= RN_MAX && 2 * RN + 2 <= W && 2 * RN + 2 <= H && !fp.point_mode;
    if (fast) {
        switch (RN) {
            case 0: transport_body<0, POW2>(sm, A, U, Anext, c, C, W, H, fp, out); break;
            case 1: transport_body<1, POW2>(sm, A, U, Anext, c, C, W, H, fp, out); break;
            case 2: transport_body<2, POW2>(sm, A, U, Anext, c, C, W, H, fp, out); break;
            default: transport_body<3, POW2>(sm, A, U, Anext, c, C, W, H, fp, out); break;
        }
    } else {
        const int Y = y0 + ty;
        const int R = RN + 1;
#pragma unroll 1
        for (int i = 0; i < 4; ++i) {
            const int X = x0 + 4 * tx + i;
            if (X < W && Y < H) {
                out[i] = gather_generic_2d(A, U, c, C, W, H, X, Y, R, fp);
                Anext[size_t(c) * N + size_t(Y) * W + X] = out[i];
            }
        }
    }
    // Spread of this channel of the next state, for the next step's window.
    float vmax = -INFINITY, vmin = INFINITY;
    bool bad = false;
    const int Y = y0 + ty;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int X = x0 + 4 * tx + i;
        if (X < W && Y < H) {
            float v = out[i];
            bad |= !isfinite(v);
            vmax = fmaxf(vmax, v);
            vmin = fminf(vmin, v);
        }
    }
    if (bound_out) block_minmax_atomic(vmax, vmin, bad, bound_out + 2 * c);
}

void launch_transport_2d(const float* A, const float* U, float* Anext, int C, int W, int H, const FlowParams& fp,
                         const int* bound_in, int* bound_out, int* status, cudaStream_t st) {
    dim3 grid((W + TT_W - 1) / TT_W, (H + TT_H - 1) / TT_H, C);
    size_t smem = transport_smem_bytes();
    if (fp.area_pow2)
        transport_2d<true><<<grid, 256, smem, st>>>(A, U, Anext, C, W, H, fp, bound_in, bound_out, status);
    else
        transport_2d<false><<<grid, 256, smem, st>>>(A, U, Anext, C, W, H, fp, bound_in, bound_out, status);
}

void transport_2d_set_attributes() {
    cudaFuncSetAttribute(transport_2d<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(transport_smem_bytes()));
    cudaFuncSetAttribute(transport_2d<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(transport_smem_bytes()));
    cudaFuncSetAttribute(transport_2d<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(transport_2d<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(conv_direct_growth_2d, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(conv_direct_smem_bytes(MAX_DIRECT_RADIUS)));
}

// ---------------------------------------------------------------------------
// Per-channel spread of a state (initial flow bound) and slot reset.
// ---------------------------------------------------------------------------
__global__ void bound_reset_kernel(int* slot, int C) {
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        slot[2 * c] = float_to_ordered(-INFINITY);
        slot[2 * c + 1] = float_to_ordered(INFINITY);
    }
}

__global__ void __launch_bounds__(256) channel_minmax(const float* __restrict__ A, size_t N, int* slot) {
    const int c = blockIdx.y;
    const float* a = A + size_t(c) * N;
    float vmax = -INFINITY, vmin = INFINITY;
    bool bad = false;
    for (size_t i = blockIdx.x * size_t(256) + threadIdx.x; i < N; i += size_t(gridDim.x) * 256) {
        float v = a[i];
        bad |= !isfinite(v);
        vmax = fmaxf(vmax, v);
        vmin = fminf(vmin, v);
    }
    block_minmax_atomic(vmax, vmin, bad, slot + 2 * c);
}

void launch_bound_reset(int* slot, int C, cudaStream_t st) {
    if (slot && C > 0) bound_reset_kernel<<<1, 32, 0, st>>>(slot, C);
}

void launch_bound_init(const float* A, int C, size_t N, int* slot, cudaStream_t st) {
    launch_bound_reset(slot, C, st);
    size_t want = (N + 255) / 256;
    int blocks = int(want < size_t(148) ? want : size_t(148));
    if (blocks > 0 && C > 0) channel_minmax<<<dim3(blocks, C), 256, 0, st>>>(A, N, slot);
}

// ---------------------------------------------------------------------------
// FP64 compensated (Neumaier) mass reduction, deterministic two-pass.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void neumaier_add(double& s, double& c, double x) {
    double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

__device__ __forceinline__ void neumaier_merge(double& s, double& c, double s2, double c2) {
    neumaier_add(s, c, s2);
    c += c2;
}

// Block merge in thread order (deterministic); the result is valid in thread 0.
__device__ void block_neumaier(double& s, double& c) {
    __shared__ double ss[256], cs[256];
    ss[threadIdx.x] = s;
    cs[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x < 32) {
        double S = ss[threadIdx.x * 8], Cc = cs[threadIdx.x * 8];
        for (int i = 1; i < 8; ++i) neumaier_merge(S, Cc, ss[threadIdx.x * 8 + i], cs[threadIdx.x * 8 + i]);
        ss[threadIdx.x * 8] = S;
        cs[threadIdx.x * 8] = Cc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = ss[0], Cc = cs[0];
        for (int w = 1; w < 32; ++w) neumaier_merge(S, Cc, ss[w * 8], cs[w * 8]);
        s = S;
        c = Cc;
    }
}

__global__ void __launch_bounds__(256) mass_partial(const float* __restrict__ A, size_t n, double2* partial) {
    double s = 0.0, c = 0.0;
    for (size_t i = blockIdx.x * size_t(256) + threadIdx.x; i < n; i += size_t(gridDim.x) * 256)
        neumaier_add(s, c, double(A[i]));
    block_neumaier(s, c);
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(s, c);
}

__global__ void __launch_bounds__(256) mass_final(const double2* partial, int np, double* out) {
    double s = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < np; i += 256) neumaier_merge(s, c, partial[i].x, partial[i].y);
    block_neumaier(s, c);
    if (threadIdx.x == 0) out[0] = s + c;
}

void launch_mass_fp64(const float* A, size_t n, double2* partial, int np, double* out, cudaStream_t st) {
    mass_partial<<<np, 256, 0, st>>>(A, n, partial);
    mass_final<<<1, 256, 0, st>>>(partial, np, out);
}

}  // namespace flp
