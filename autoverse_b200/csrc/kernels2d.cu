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
                                                             int* reset_slot) {
    extern __shared__ float sm[];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * 32 + tx;
    const int c = blockIdx.z;
    const int x0 = blockIdx.x * CD_TW, y0 = blockIdx.y * CD_TH;
    const size_t N = size_t(W) * H;
    if (reset_slot && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && tid == 0) {
        reset_slot[0] = float_to_ordered(-INFINITY);
        reset_slot[1] = float_to_ordered(INFINITY);
    }
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
    conv_direct_growth_2d<<<grid, dim3(32, 8), smem, st>>>(A, U, kd, K, taps, W, H, rmax, reset_slot);
}

// ---------------------------------------------------------------------------
// Gather radius from the flow bound.
// |F_x|,|F_y| <= max(max|grad U|, max|grad A_sum|) since F = (1-a)gU - a gA
// with a in [0,1]; the Sobel/8 of a field ranges over at most half its spread,
// |U| <= sum_k |w_k| (G in [-1,1]) and A_sum spans [amin, amax].  A source
// at x can deposit only into cells ix with |ix - x| < dt|F| + s + 1.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int gather_radius(const int* bound, const FlowParams& fp, int maxside, int* status) {
    float amax = ordered_to_float(bound[0]);
    float amin = ordered_to_float(bound[1]);
    float spread = amax - amin;
    if (!(spread >= 0.f) || !isfinite(spread)) {
        if (status && threadIdx.x == 0 && threadIdx.y == 0) atomicOr(status, STATUS_NONFINITE);
        return 1;
    }
    float fb = fmaxf(fp.ubound, 0.5f * spread);
    float Db = fp.dt * fb * 1.0001f + 1e-5f;
    float rr = floorf(Db + fp.s + 1.0f);
    int cap = 2 * maxside + 2;
    if (!(rr < float(cap))) return cap;
    return rr < 1.f ? 1 : int(rr);
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
// Fused transport: tile 64x32 destinations, 256 threads; thread (tx, ty)
// owns the 4-cell row strips at (x0+4tx.., y0+ty) and (x0+4tx.., y0+ty+16).
// Source region = tile + TP cells each side (TP = widest fast-path radius).
// ---------------------------------------------------------------------------
constexpr int TT_W = 64, TT_H = 32, TP = 4;
constexpr int SR_W = TT_W + 2 * TP, SR_H = TT_H + 2 * TP;  // 72 x 40 sources
constexpr int AR_W = SR_W + 2, AR_H = SR_H + 2;            // 74 x 42 with the Sobel ring

size_t transport_smem_bytes() { return sizeof(float) * (2 * AR_W * AR_H + 3 * SR_W * SR_H); }

__device__ __forceinline__ int wrap_pass(int g, int size) { return g >= size ? 0 : (g < 0 ? 2 : 1); }

__device__ __forceinline__ void block_minmax_atomic(float vmax, float vmin, int* slot) {
    __shared__ float red_max[8], red_min[8];
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
        // NaN propagates into the slot as a non-finite spread the next step detects.
        if (mx != mx || mn != mn) { mx = NAN; mn = NAN; }
        atomicMax(slot + 0, float_to_ordered(mx));
        atomicMin(slot + 1, float_to_ordered(mn));
    }
}

template <bool POW2>
__global__ void __launch_bounds__(256) transport_2d(const float* __restrict__ A, const float* __restrict__ U,
                                                    float* __restrict__ Anext, int C, int W, int H, FlowParams fp,
                                                    const int* __restrict__ bound_in, int* bound_out, int* status) {
    extern __shared__ float sm[];
    float* asum = sm;                   // AR_H x AR_W
    float* usm = asum + AR_W * AR_H;    // AR_H x AR_W
    float* dxs = usm + AR_W * AR_H;     // SR_H x SR_W
    float* dys = dxs + SR_W * SR_H;
    float* mss = dys + SR_W * SR_H;

    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TT_W, y0 = blockIdx.y * TT_H;
    const size_t N = size_t(W) * H;
    const int R = gather_radius(bound_in, fp, max(W, H), status);

    float nsum[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int i = 0; i < 4; ++i) nsum[h][i] = 0.f;

    const bool fast = R <= TP && 2 * R + 1 <= W && 2 * R + 1 <= H && !fp.point_mode;
    if (!fast) {
        for (int c = 0; c < C; ++c)
            for (int h = 0; h < 2; ++h) {
                int Y = y0 + ty + 16 * h;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    int X = x0 + 4 * tx + i;
                    if (X < W && Y < H) {
                        float v = gather_generic_2d(A, U, c, C, W, H, X, Y, R, fp);
                        Anext[size_t(c) * N + size_t(Y) * W + X] = v;
                        nsum[h][i] = __fadd_rn(nsum[h][i], v);
                    }
                }
            }
    } else {
        // Channel sum over the source region plus the Sobel ring.
        for (int i = tid; i < AR_W * AR_H; i += 256) {
            int ly = i / AR_W, lx = i - ly * AR_W;
            int gy = wrap_coord(y0 - TP - 1 + ly, H), gx = wrap_coord(x0 - TP - 1 + lx, W);
            size_t idx = size_t(gy) * W + gx;
            float s = 0.f;
            for (int c = 0; c < C; ++c) s = __fadd_rn(s, A[size_t(c) * N + idx]);
            asum[i] = s;
        }
        // Which wrap passes occur for this tile (block-uniform).
        const int rp_lo = (y0 + TT_H - 1 + R >= H) ? 0 : 1, rp_hi = (y0 - R < 0) ? 2 : 1;
        const int cp_lo = (x0 + TT_W - 1 + R >= W) ? 0 : 1, cp_hi = (x0 - R < 0) ? 2 : 1;
        const float s = fp.s;

        for (int c = 0; c < C; ++c) {
            const float* Ac = A + size_t(c) * N;
            const float* Uc = U + size_t(c) * N;
            __syncthreads();
            for (int i = tid; i < AR_W * AR_H; i += 256) {
                int ly = i / AR_W, lx = i - ly * AR_W;
                int gy = wrap_coord(y0 - TP - 1 + ly, H), gx = wrap_coord(x0 - TP - 1 + lx, W);
                usm[i] = Uc[size_t(gy) * W + gx];
            }
            __syncthreads();
            // Per-source destination (reintegration.rs:81-82) and mass.
            for (int i = tid; i < SR_W * SR_H; i += 256) {
                int sy = i / SR_W, sx = i - sy * SR_W;
                int yw = wrap_coord(y0 - TP + sy, H), xw = wrap_coord(x0 - TP + sx, W);
                float mass = Ac[size_t(yw) * W + xw];
                if (fabsf(mass) < 1e-10f) mass = 0.f;
                const float* a = asum + sy * AR_W + sx;  // top-left of the 3x3 window
                const float* u = usm + sy * AR_W + sx;
                float gax, gay, gux, guy;
                sobel2(a[0], a[1], a[2], a[AR_W], a[AR_W + 2], a[2 * AR_W], a[2 * AR_W + 1], a[2 * AR_W + 2], gax, gay);
                sobel2(u[0], u[1], u[2], u[AR_W], u[AR_W + 2], u[2 * AR_W], u[2 * AR_W + 1], u[2 * AR_W + 2], gux, guy);
                float alpha = flow_alpha(a[AR_W + 1], fp.beta_a, fp.nexp);
                float oma = __fsub_rn(1.0f, alpha);
                float fx = __fsub_rn(__fmul_rn(oma, gux), __fmul_rn(alpha, gax));
                float fy = __fsub_rn(__fmul_rn(oma, guy), __fmul_rn(alpha, gay));
                dxs[i] = __fadd_rn(float(xw), __fmul_rn(fp.dt, fx));
                dys[i] = __fadd_rn(float(yw), __fmul_rn(fp.dt, fy));
                mss[i] = mass;
            }
            __syncthreads();
            // Gather.
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const int Y = y0 + ty + 16 * h;
                const int X0 = x0 + 4 * tx;
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                if (Y < H && X0 < W) {
#pragma unroll 1
                    for (int rp = rp_lo; rp <= rp_hi; ++rp) {
#pragma unroll 1
                        for (int ky = -R; ky <= R; ++ky) {
                            const int gy = Y + ky;
                            if (wrap_pass(gy, H) != rp) continue;
                            const int iy = Y + (gy < 0 ? H : (gy >= H ? -H : 0));
                            const float cy0 = float(iy), cy1 = float(iy + 1);
                            const int sr = (Y - y0) + TP + ky;
                            const float4* rx = reinterpret_cast<const float4*>(dxs + sr * SR_W + 4 * tx);
                            const float4* ry = reinterpret_cast<const float4*>(dys + sr * SR_W + 4 * tx);
                            const float4* rm = reinterpret_cast<const float4*>(mss + sr * SR_W + 4 * tx);
                            float vx[12], vy[12], vm[12];
#pragma unroll
                            for (int q = 0; q < 3; ++q) {
                                float4 a4 = rx[q], b4 = ry[q], m4 = rm[q];
                                vx[4 * q] = a4.x; vx[4 * q + 1] = a4.y; vx[4 * q + 2] = a4.z; vx[4 * q + 3] = a4.w;
                                vy[4 * q] = b4.x; vy[4 * q + 1] = b4.y; vy[4 * q + 2] = b4.z; vy[4 * q + 3] = b4.w;
                                vm[4 * q] = m4.x; vm[4 * q + 1] = m4.y; vm[4 * q + 2] = m4.z; vm[4 * q + 3] = m4.w;
                            }
#pragma unroll 1
                            for (int cp = cp_lo; cp <= cp_hi; ++cp) {
#pragma unroll
                                for (int j = 0; j < 12; ++j) {
                                    const int gx = x0 - TP + 4 * tx + j;
                                    if (wrap_pass(gx, W) != cp) continue;
                                    const float m = vm[j];
                                    if (m == 0.f) continue;
                                    const float ymin = __fsub_rn(vy[j], s), ymax = __fadd_rn(vy[j], s);
                                    const float oy0 = fmaxf(cy0, ymin), oy1 = fminf(cy1, ymax);
                                    const float oh = fmaxf(__fsub_rn(oy1, oy0), 0.f);
                                    if (!(oh > 0.f)) continue;
                                    const float xmin = __fsub_rn(vx[j], s), xmax = __fadd_rn(vx[j], s);
                                    const int xsh = gx < 0 ? W : (gx >= W ? -W : 0);
#pragma unroll
                                    for (int i = 0; i < 4; ++i) {
                                        const int X = X0 + i;
                                        const int kx = gx - X;
                                        if (kx < -R || kx > R) continue;
                                        const int ix = X + xsh;
                                        const float ox0 = fmaxf(float(ix), xmin), ox1 = fminf(float(ix + 1), xmax);
                                        const float ow = fmaxf(__fsub_rn(ox1, ox0), 0.f);
                                        const float area = __fmul_rn(ow, oh);
                                        if (area > 0.f) {
                                            const float frac = POW2 ? __fmul_rn(area, fp.inv_area)
                                                                    : __fdiv_rn(area, fp.total_area);
                                            acc[i] = __fadd_rn(acc[i], __fmul_rn(m, frac));
                                        }
                                    }
                                }
                            }
                        }
                    }
                    float* out = Anext + size_t(c) * N + size_t(Y) * W;
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        if (X0 + i < W) {
                            out[X0 + i] = acc[i];
                            nsum[h][i] = __fadd_rn(nsum[h][i], acc[i]);
                        }
                    }
                }
            }
        }
    }
    // Spread of the next channel sum, for the next step's gather radius.
    float vmax = -INFINITY, vmin = INFINITY;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int X = x0 + 4 * tx + i, Y = y0 + ty + 16 * h;
            if (X < W && Y < H) {
                float v = nsum[h][i];
                if (v != v) { vmax = NAN; vmin = NAN; }
                else { vmax = fmaxf(vmax, v); vmin = fminf(vmin, v); }
            }
        }
    if (bound_out) block_minmax_atomic(vmax, vmin, bound_out);
}

void launch_transport_2d(const float* A, const float* U, float* Anext, int C, int W, int H, const FlowParams& fp,
                         const int* bound_in, int* bound_out, int* status, cudaStream_t st) {
    dim3 grid((W + TT_W - 1) / TT_W, (H + TT_H - 1) / TT_H);
    size_t smem = transport_smem_bytes();
    if (fp.area_pow2)
        transport_2d<true><<<grid, 256, smem, st>>>(A, U, Anext, C, W, H, fp, bound_in, bound_out, status);
    else
        transport_2d<false><<<grid, 256, smem, st>>>(A, U, Anext, C, W, H, fp, bound_in, bound_out, status);
}

void transport_2d_set_attributes() {
    cudaFuncSetAttribute(transport_2d<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(transport_smem_bytes()));
    cudaFuncSetAttribute(transport_2d<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(transport_smem_bytes()));
    cudaFuncSetAttribute(conv_direct_growth_2d, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(conv_direct_smem_bytes(MAX_DIRECT_RADIUS)));
}

// ---------------------------------------------------------------------------
// Spread of the channel sum of a state (initial flow bound).
// ---------------------------------------------------------------------------
__global__ void bound_reset_kernel(int* slot) {
    slot[0] = float_to_ordered(-INFINITY);
    slot[1] = float_to_ordered(INFINITY);
}

__global__ void __launch_bounds__(256) channel_sum_minmax(const float* __restrict__ A, int C, size_t N, int* slot) {
    float vmax = -INFINITY, vmin = INFINITY;
    for (size_t i = blockIdx.x * size_t(256) + threadIdx.x; i < N; i += size_t(gridDim.x) * 256) {
        float s = 0.f;
        for (int c = 0; c < C; ++c) s = __fadd_rn(s, A[size_t(c) * N + i]);
        if (s != s) { vmax = NAN; vmin = NAN; break; }
        vmax = fmaxf(vmax, s);
        vmin = fminf(vmin, s);
    }
    block_minmax_atomic(vmax, vmin, slot);
}

void launch_bound_reset(int* slot, cudaStream_t st) {
    if (slot) bound_reset_kernel<<<1, 1, 0, st>>>(slot);
}

void launch_bound_init(const float* A, int C, size_t N, int* slot, cudaStream_t st) {
    bound_reset_kernel<<<1, 1, 0, st>>>(slot);
    size_t want = (N + 255) / 256;
    int blocks = int(want < size_t(148 * 4) ? want : size_t(148 * 4));
    if (blocks > 0 && C > 0) channel_sum_minmax<<<blocks, 256, 0, st>>>(A, C, N, slot);
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
