// 3D transport kernels (replace CpuPropagator3D::step's stencil and
// reintegration, src/compute/propagator3d.rs:181-256):
//   * flow_3d — channel sum, the 3x3x3 Sobel of the sum and of U_c in the
//     reference's evaluation order (gradient3d.rs:106-138), alpha, the flow
//     F = (1-a) grad U - a grad A (flow3d.rs:64-72) and dest = x + dt*F
//     (reintegration3d.rs:82-84), one thread per cell;
//   * gather_3d — cube reintegration in gather form (reintegration3d.rs:109-198):
//     each destination sums the overlap volumes of the sources in the window
//     [-RN, RN+1]^3 in the reference's deposit order (z, then y, then x over
//     wrapped source indices), bit-identical to the reference's scatter.
#include "common.cuh"
#include "kernels.h"
#include "transport_items.cuh"

namespace flp {

// ------------------------------------------------------------- flow_3d ----
// A CTA owns a 32x8 block of columns in NZ consecutive planes and stages the
// NZ + 2 planes of A, U and the channel sum that their stencils read: NZ = 4
// when those blocks fit one CTA's shared memory (up to 13 channels; fewer
// halo planes per output plane), else NZ = 2 (up to 20 channels).
constexpr int F3_W = 32, F3_H = 8;
constexpr int F3_RW = F3_W + 2, F3_RH = F3_H + 2, F3_PL = F3_RW * F3_RH;
__host__ __device__ constexpr int f3_rc(int nz) { return (nz + 2) * F3_PL; }  // floats of one staged block
constexpr size_t F3_SMEM_MAX = 227 * 1024 - 1024;  // a CTA's 227 KB less room for the static arrays

size_t flow3d_smem_bytes(int C, int nz) { return sizeof(float) * (size_t(2 * C + 1) * f3_rc(nz)); }
static int flow3d_nz(int C) { return flow3d_smem_bytes(C, 4) <= F3_SMEM_MAX ? 4 : 2; }
// Channels whose staged A and U blocks plus the channel sum fit one CTA's
// shared memory with two planes per CTA.
int flow3d_max_channels() { return int((F3_SMEM_MAX / (sizeof(float) * f3_rc(2)) - 1) / 2); }

// 3D Sobel of a field at the centre of a 3x3x3 window w[z][y][x] (region
// indices), gradient3d.rs:106-138: each line sum (a + 2b) + c, each gradient
// ((l_m + 2 l_0) + l_p) / 32, all in f32 without contraction.
struct Win3 {
    const float* p;  // element (dz, dy, dx) at p[dz*F3_PL + dy*F3_RW + dx], dz in 0..NZ+1, dy,dx in 0..2
    __device__ float at(int z, int y, int x) const { return p[z * F3_PL + y * F3_RW + x]; }
};
__device__ __forceinline__ float line3(float a, float b, float c) { return __fadd_rn(__fadd_rn(a, __fmul_rn(2.0f, b)), c); }
__device__ __forceinline__ float diff3(float lm, float lp) { return __fadd_rn(-lm, lp); }
__device__ __forceinline__ float comb3(float m, float z, float p) {
    return __fmul_rn(__fadd_rn(__fadd_rn(m, __fmul_rn(2.0f, z)), p), 0.03125f);
}

// The Sobel gradients of the NZ windows that start at layers 0..NZ-1 of an
// (NZ+2)-layer block (cells at layers 1..NZ).  Per layer z the column sums
// over y, Ly[z][x] = line3(w(z,0,x), w(z,1,x), w(z,2,x)), and the row sums
// over x, Lx[z][y] = line3(w(z,y,0), w(z,y,1), w(z,y,2)), are formed once;
// the reference's terms are exactly these:
//   x gradient: per layer diff3(Ly[z][0], Ly[z][2]), combined over the window's layers;
//   y gradient: per layer diff3(Lx[z][0], Lx[z][2]), combined over the window's layers;
//   z gradient: per column diff3(Ly[first][x], Ly[last][x]), combined over x.
template <int NZ>
__device__ __forceinline__ void sobel3_run(const Win3& w, float (&gx)[NZ], float (&gy)[NZ], float (&gz)[NZ]) {
    constexpr int NL = NZ + 2;
    float ly[NL][3], dx[NL], dy[NL];
#pragma unroll
    for (int z = 0; z < NL; ++z) {
#pragma unroll
        for (int x = 0; x < 3; ++x) ly[z][x] = line3(w.at(z, 0, x), w.at(z, 1, x), w.at(z, 2, x));
        dx[z] = diff3(ly[z][0], ly[z][2]);
        dy[z] = diff3(line3(w.at(z, 0, 0), w.at(z, 0, 1), w.at(z, 0, 2)), line3(w.at(z, 2, 0), w.at(z, 2, 1), w.at(z, 2, 2)));
    }
#pragma unroll
    for (int k = 0; k < NZ; ++k) {
        gx[k] = comb3(dx[k], dx[k + 1], dx[k + 2]);
        gy[k] = comb3(dy[k], dy[k + 1], dy[k + 2]);
        gz[k] = comb3(diff3(ly[k][0], ly[k + 2][0]), diff3(ly[k][1], ly[k + 2][1]), diff3(ly[k][2], ly[k + 2][2]));
    }
}

template <int F3_NZ>
__global__ void __launch_bounds__(256) flow_3d(const float* __restrict__ A, const float* __restrict__ U,
                                               float* __restrict__ DX, float* __restrict__ DY,
                                               float* __restrict__ DZ, int C, int W, int H, int D, FlowParams fp,
                                               int* dmax_slot, int* status) {
    dep_enter();
    constexpr int F3_NP = F3_NZ + 2, F3_RC = f3_rc(F3_NZ);
    extern __shared__ __align__(16) float sm[];
    float* as = sm;                    // C staged A blocks (F3_NP planes each)
    float* us = sm + C * F3_RC;        // C staged U blocks
    float* asum = sm + 2 * C * F3_RC;  // channel sum
    __shared__ int colx[F3_RW], rowy[F3_RH], plz[F3_NP];
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * F3_W, y0 = blockIdx.y * F3_H, z0 = blockIdx.z * F3_NZ;
    const size_t N = size_t(W) * H * D;
    if (tid < F3_RW) colx[tid] = wrap_near(x0 - 1 + tid, W);
    else if (tid < F3_RW + F3_RH) rowy[tid - F3_RW] = wrap_near(y0 - 1 + (tid - F3_RW), H);
    else if (tid < F3_RW + F3_RH + F3_NP) plz[tid - F3_RW - F3_RH] = wrap_near(z0 - 1 + (tid - F3_RW - F3_RH), D);
    __syncthreads();
    // one staged row (field k, plane pz, row ly) per warp and pass, lanes over
    // its 34 columns: no index division per element
    {
        const int lane = tid & 31, warp = tid >> 5;
        const int x_a = colx[lane], x_b = lane < F3_RW - 32 ? colx[32 + lane] : 0;
        for (int row = warp; row < 2 * C * F3_NP * F3_RH; row += 8) {
            const int k = row / (F3_NP * F3_RH), q = row - k * (F3_NP * F3_RH);
            const int pz = q / F3_RH, ly = q - pz * F3_RH;
            const float* src = (k < C ? A + size_t(k) * N : U + size_t(k - C) * N) +
                               (size_t(plz[pz]) * H + rowy[ly]) * W;
            float* dst = sm + k * F3_RC + pz * F3_PL + ly * F3_RW;
            cp_async4(dst + lane, src + x_a);
            if (lane < F3_RW - 32) cp_async4(dst + 32 + lane, src + x_b);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    for (int i = tid; i < F3_RC; i += 256) {
        float a = 0.f;
        for (int k = 0; k < C; ++k) a = __fadd_rn(a, as[k * F3_RC + i]);
        asum[i] = a;
    }
    __syncthreads();
    const int lx = tid & (F3_W - 1), ly = tid / F3_W;
    const int X = x0 + lx, Y = y0 + ly;
    // Depths are the z-transform sizes (multiples of 16), so every plane block
    // is full; the bound only guards the stores.
    const int nz = min(F3_NZ, D - z0);
    float dmax = 0.f;
    bool bad = false;
    if (X < W && Y < H) {
        const int o = ly * F3_RW + lx;  // (0,0,0) corner of the first window
        float gax[F3_NZ], gay[F3_NZ], gaz[F3_NZ], oma[F3_NZ], agx[F3_NZ], agy[F3_NZ], agz[F3_NZ];
        sobel3_run<F3_NZ>(Win3{asum + o}, gax, gay, gaz);
#pragma unroll
        for (int k = 0; k < F3_NZ; ++k) {
            const float alpha = alpha_fp(asum[(k + 1) * F3_PL + o + F3_RW + 1], fp);
            oma[k] = __fsub_rn(1.0f, alpha);
            agx[k] = __fmul_rn(alpha, gax[k]);
            agy[k] = __fmul_rn(alpha, gay[k]);
            agz[k] = __fmul_rn(alpha, gaz[k]);
        }
        for (int c = 0; c < C; ++c) {
            float gux[F3_NZ], guy[F3_NZ], guz[F3_NZ];
            sobel3_run<F3_NZ>(Win3{us + c * F3_RC + o}, gux, guy, guz);
#pragma unroll
            for (int k = 0; k < F3_NZ; ++k) {
                if (k >= nz) break;
                const int z = z0 + k;
                const size_t cell = (size_t(z) * H + Y) * W + X;
                const float fx = __fsub_rn(__fmul_rn(oma[k], gux[k]), agx[k]);
                const float fy = __fsub_rn(__fmul_rn(oma[k], guy[k]), agy[k]);
                const float fz = __fsub_rn(__fmul_rn(oma[k], guz[k]), agz[k]);
                const float dx = __fadd_rn(float(X), __fmul_rn(fp.dt, fx));
                const float dy = __fadd_rn(float(Y), __fmul_rn(fp.dt, fy));
                const float dz = __fadd_rn(float(z), __fmul_rn(fp.dt, fz));
                const float mass = as[c * F3_RC + (k + 1) * F3_PL + o + F3_RW + 1];
                bad |= !(isfinite(mass) && isfinite(dx) && isfinite(dy) && isfinite(dz));
                if (fabsf(mass) >= 1e-10f)
                    dmax = fmaxf(dmax, fmaxf(fabsf(dx - float(X)), fmaxf(fabsf(dy - float(Y)), fabsf(dz - float(z)))));
                DX[size_t(c) * N + cell] = dx;
                DY[size_t(c) * N + cell] = dy;
                DZ[size_t(c) * N + cell] = dz;
            }
        }
    }
    if (status && __syncthreads_or(bad ? 1 : 0) && tid == 0) atomicOr(status, STATUS_NONFINITE);
    block_max_atomic(dmax, bad, dmax_slot);
}

// ----------------------------------------------------------- gather_3d ----
constexpr int G3_W = 32, G3_H = 8, G3_RNMAX = 2;
constexpr int G3_SW = G3_W + 2 * G3_RNMAX + 1, G3_SH = G3_H + 2 * G3_RNMAX + 1, G3_SD = 2 * G3_RNMAX + 2;
constexpr int G3_CELLS = G3_SW * G3_SH * G3_SD;



// Overlap of one source cube with cell (ix, iy, iz): reintegration3d.rs:155-185.
template <bool POW2>
__device__ __forceinline__ float cube_term(float m, float dx, float dy, float dz, int ix, int iy, int iz,
                                           const FlowParams& fp) {
    const float s = fp.s;
    const float ox0 = fmaxf(float(ix), __fsub_rn(dx, s)), ox1 = fminf(float(ix + 1), __fadd_rn(dx, s));
    const float oy0 = fmaxf(float(iy), __fsub_rn(dy, s)), oy1 = fminf(float(iy + 1), __fadd_rn(dy, s));
    const float oz0 = fmaxf(float(iz), __fsub_rn(dz, s)), oz1 = fminf(float(iz + 1), __fadd_rn(dz, s));
    const float ow = fmaxf(__fsub_rn(ox1, ox0), 0.f);
    const float oh = fmaxf(__fsub_rn(oy1, oy0), 0.f);
    const float od = fmaxf(__fsub_rn(oz1, oz0), 0.f);
    const float vol = __fmul_rn(__fmul_rn(ow, oh), od);
    if (POW2) return __fmul_rn(m, vol);  // m holds mass / total_volume (exact); a zero volume adds a signed zero
    if (!(vol > 0.f)) return 0.f;
    return __fmul_rn(m, __fdiv_rn(vol, fp.total_area));
}

// Offsets k in the window [-RN, RN+1] (NW = 2RN+2 of them) in the order that
// makes the wrapped coordinates (c + k) mod size ascend; valid when NW <= size.
__device__ __forceinline__ int rot_window(int j, int c, int RN, int size) {
    const int NW = 2 * RN + 2;
    const int n_hi = max(0, c + RN + 2 - size);  // k with c + k >= size
    const int n_lo = max(0, RN - c);             // k with c + k < 0
    if (j < n_hi) return RN + 2 - n_hi + j;
    if (j < NW - n_lo) return -RN + n_lo + (j - n_hi);
    return -RN + (j - (NW - n_lo));
}

// rot_window as a rotation: offset j of the wrapped-ascending order is the
// natural offset (j + r) mod NW (natural index i = k + RN).  At most one of
// n_hi and n_lo is nonzero when NW <= size.
__device__ __forceinline__ int window_rotation(int c, int RN, int size) {
    const int NW = 2 * RN + 2;
    const int n_hi = max(0, c + RN + 2 - size);
    const int n_lo = max(0, RN - c);
    return n_lo > 0 ? n_lo : (NW - n_hi) % NW;
}

// t[j] <- t[(j + r) mod NW] with selects only (NW a power of two, 0 <= r < NW).
template <int NW>
__device__ __forceinline__ void rotate_left(float (&t)[NW], int r) {
    static_assert((NW & (NW - 1)) == 0, "window width must be a power of two");
#pragma unroll
    for (int b = 1; b < NW; b <<= 1) {
        const bool on = (r & b) != 0;
        float u[NW];
#pragma unroll
        for (int j = 0; j < NW; ++j) u[j] = on ? t[(j + b) % NW] : t[j];
#pragma unroll
        for (int j = 0; j < NW; ++j) t[j] = u[j];
    }
}

// One 32x8 block of destinations in plane Z of one channel.
template <int RN, bool POW2>
__device__ void gather3d_plane(float* sm, const float* __restrict__ DX, const float* __restrict__ DY,
                               const float* __restrict__ DZ, const float* __restrict__ A, float* __restrict__ out,
                               int W, int H, int D, int Z, const FlowParams& fp) {
    constexpr int SW = G3_W + 2 * RN + 1, SH = G3_H + 2 * RN + 1, SD = 2 * RN + 2, PL = SW * SH, NC = PL * SD;
    float* sx = sm;
    float* sy = sx + NC;
    float* sz = sy + NC;
    float* smm = sz + NC;
    __shared__ int colx[G3_SW], rowy[G3_SH], plz[G3_SD];
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * G3_W, y0 = blockIdx.y * G3_H;
    if (tid < SW) colx[tid] = wrap_near(x0 - RN + tid, W);
    else if (tid < SW + SH) rowy[tid - SW] = wrap_near(y0 - RN + (tid - SW), H);
    else if (tid < SW + SH + SD) plz[tid - SW - SH] = wrap_near(Z - RN + (tid - SW - SH), D);
    __syncthreads();
    for (int i = tid; i < 4 * NC; i += 256) {
        const int k = i / NC, cell = i - k * NC;
        const int pz = cell / PL, r = cell - pz * PL;
        const int ly = r / SW, lx = r - ly * SW;
        const size_t idx = (size_t(plz[pz]) * H + rowy[ly]) * W + colx[lx];
        const float* src = k == 0 ? DX : (k == 1 ? DY : (k == 2 ? DZ : A));
        cp_async4(sm + i, src + idx);
    }
    cp_async_wait_all();
    __syncthreads();
    for (int i = tid; i < NC; i += 256) smm[i] = source_mass<POW2>(smm[i], fp);  // state -> source mass
    __syncthreads();
    const int lx = tid & (G3_W - 1), ly = tid / G3_W;
    const int X = x0 + lx, Y = y0 + ly;
    if (X >= W || Y >= H) return;
    float acc = 0.f;
    // Offsets k = source - destination in [-RN, RN+1] per axis, visited so the
    // wrapped source indices ascend (z outer, then y, then x).
    constexpr int NW = 2 * RN + 2;
    for (int jz = 0; jz < NW; ++jz) {
        const int kz = rot_window(jz, Z, RN, D);
        const int gz = Z + kz;
        const int iz = Z + (gz < 0 ? D : (gz >= D ? -D : 0));
        for (int jy = 0; jy < NW; ++jy) {
            const int ky = rot_window(jy, Y, RN, H);
            const int gy = Y + ky;
            const int iy = Y + (gy < 0 ? H : (gy >= H ? -H : 0));
            const int rowbase = (kz + RN) * PL + (ly + ky + RN) * SW;
#pragma unroll
            for (int jx = 0; jx < NW; ++jx) {
                const int kx = rot_window(jx, X, RN, W);
                const int gx = X + kx;
                const int ix = X + (gx < 0 ? W : (gx >= W ? -W : 0));
                const int o = rowbase + lx + kx + RN;
                const float m = smm[o];
                if (!POW2 && m == 0.f) continue;
                acc = __fadd_rn(acc, cube_term<POW2>(m, sx[o], sy[o], sz[o], ix, iy, iz, fp));
            }
        }
    }
    out[(size_t(Z) * H + Y) * W + X] = acc;
}

// Generic per-destination gather from global memory for any window; also the
// nearest-cell mode and the reference's [-W, 2W] cell clamps.
template <bool POW2>
__device__ float gather3d_generic(const float* __restrict__ DX, const float* __restrict__ DY,
                                  const float* __restrict__ DZ, const float* __restrict__ A, int W, int H, int D,
                                  int X, int Y, int Z, int R, const FlowParams& fp) {
    float acc = 0.f;
    for (int jz = 0; jz <= 2 * R; ++jz) {
        const int kz = rotated_offset(jz, Z, R, D);
        const int zw = wrap_coord(Z + kz, D), iz = zw - kz;
        for (int jy = 0; jy <= 2 * R; ++jy) {
            const int ky = rotated_offset(jy, Y, R, H);
            const int yw = wrap_coord(Y + ky, H), iy = yw - ky;
            for (int jx = 0; jx <= 2 * R; ++jx) {
                const int kx = rotated_offset(jx, X, R, W);
                const int xw = wrap_coord(X + kx, W), ix = xw - kx;
                const size_t src = (size_t(zw) * H + yw) * W + xw;
                const float m = source_mass<POW2>(A[src], fp);
                if (m == 0.f) continue;
                const float dx = DX[src], dy = DY[src], dz = DZ[src];
                if (fp.point_mode) {
                    if (f2i_sat(roundf(dx)) == ix && f2i_sat(roundf(dy)) == iy && f2i_sat(roundf(dz)) == iz)
                        acc = __fadd_rn(acc, m);
                    continue;
                }
                const float s = fp.s;
                const int ix_lo = max(f2i_sat(floorf(__fsub_rn(dx, s))), -W), ix_hi = min(f2i_sat(ceilf(__fadd_rn(dx, s))), 2 * W);
                const int iy_lo = max(f2i_sat(floorf(__fsub_rn(dy, s))), -H), iy_hi = min(f2i_sat(ceilf(__fadd_rn(dy, s))), 2 * H);
                const int iz_lo = max(f2i_sat(floorf(__fsub_rn(dz, s))), -D), iz_hi = min(f2i_sat(ceilf(__fadd_rn(dz, s))), 2 * D);
                if (ix < ix_lo || ix > ix_hi || iy < iy_lo || iy > iy_hi || iz < iz_lo || iz > iz_hi) continue;
                const float t = cube_term<POW2>(m, dx, dy, dz, ix, iy, iz, fp);
                if (t != 0.f) acc = __fadd_rn(acc, t);
            }
        }
    }
    return acc;
}

// ---- z-marching gather with overlap tables (RN <= 1) ----------------------
// A CTA owns a 32x8 block of destination columns and G3_NZ consecutive
// planes.  It keeps the 2RN+2 source planes that can reach the current
// output plane in a ring in shared memory, each as per-source tables of the
// x, y and z overlaps with the 2RN+2 candidate destination coordinates
// (component k: destination = the source's own wrapped coordinate - (k - RN),
// reintegration3d.rs:155-175) and the mass.  Each output plane loads one new
// source plane.  A term is then vol = (ow * oh) * od, acc += m * vol: the
// reference's operations, added in its deposit order (z, y, x over wrapped
// source indices), with the overlap arithmetic done once per source instead
// of once per (source, destination) pair.
constexpr int G3_NZ = 8;

// With PAIRS a thread takes its column's output planes two at a time (Z and
// Z+1): a source's mass and its x and y overlaps serve both destinations and
// the first product ow * oh of its volume is shared, so a pair of terms takes
// five shared-memory loads instead of eight.  The ring then holds 2RN+3
// planes.  Pairs whose z windows wrap the torus take the planes one by one.
#ifndef FLP_GATHER3D_PAIRS
#define FLP_GATHER3D_PAIRS 1
#endif
constexpr bool G3_PAIRS = FLP_GATHER3D_PAIRS != 0;

template <int RN>
struct March3 {
    static constexpr int SW = G3_W + 2 * RN + 1, SH = G3_H + 2 * RN + 1, NS = SW * SH;
    static constexpr int NW = 2 * RN + 2, SD = 2 * RN + 2 + (G3_PAIRS ? 1 : 0);
    static constexpr int PLANE = (3 * NW + 1) * NS;  // floats per ring slot
    static constexpr size_t bytes = sizeof(float) * size_t(SD) * PLANE;
};

template <int RN, bool POW2>
__device__ void gather3d_march(float* sm, const float* __restrict__ DX, const float* __restrict__ DY,
                               const float* __restrict__ DZ, const float* __restrict__ A, float* __restrict__ out,
                               int W, int H, int D, int z0, int nz, const FlowParams& fp) {
    using M = March3<RN>;
    constexpr int SW = M::SW, SH = M::SH, NS = M::NS, NW = M::NW, SD = M::SD;
    __shared__ int colx[March3<1>::SW], rowy[March3<1>::SH];
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * G3_W, y0 = blockIdx.y * G3_H;
    if (tid < SW) colx[tid] = wrap_near(x0 - RN + tid, W);
    else if (tid < SW + SH) rowy[tid - SW] = wrap_near(y0 - RN + (tid - SW), H);
    __syncthreads();
    const float s = fp.s;
    // A source plane is fetched into registers (NSP sources per thread) one
    // output plane ahead, so its global loads are in flight while the current
    // plane is gathered, and stored as overlap tables after that.
    constexpr int NSP = (NS + 255) / 256;
    auto fetch = [&](int gz, float (&r)[4][NSP]) {  // gz: unwrapped source plane, >= z0 - RN
        const size_t zoff = size_t(wrap_near(gz, D)) * H;
#pragma unroll
        for (int p = 0; p < NSP; ++p) {
            const int i = tid + 256 * p;
            if (i < NS) {
                const int ly = i / SW, lx = i - ly * SW;
                const size_t idx = (zoff + rowy[ly]) * W + colx[lx];
                r[0][p] = DX[idx];
                r[1][p] = DY[idx];
                r[2][p] = DZ[idx];
                r[3][p] = A[idx];
            }
        }
    };
    auto slot = [&](int gz) { return sm + ((gz - (z0 - RN)) % SD) * M::PLANE; };
    auto store = [&](int gz, const float (&r)[4][NSP]) {
        float* P = slot(gz);
        float* OW = P;
        float* OH = P + NW * NS;
        float* OD = P + 2 * NW * NS;
        float* Mm = P + 3 * NW * NS;
        const int zw = wrap_near(gz, D);
#pragma unroll
        for (int p = 0; p < NSP; ++p) {
            const int i = tid + 256 * p;
            if (i < NS) {
                const int ly = i / SW, lx = i - ly * SW;
                const int xw = colx[lx], yw = rowy[ly];
                Mm[i] = source_mass<POW2>(r[3][p], fp);
                const float xa = __fsub_rn(r[0][p], s), xb = __fadd_rn(r[0][p], s);
                const float ya = __fsub_rn(r[1][p], s), yb = __fadd_rn(r[1][p], s);
                const float za = __fsub_rn(r[2][p], s), zb = __fadd_rn(r[2][p], s);
#pragma unroll
                for (int k = 0; k < NW; ++k) {
                    const int ix = xw - (k - RN), iy = yw - (k - RN), iz = zw - (k - RN);
                    OW[k * NS + i] = fmaxf(__fsub_rn(fminf(float(ix + 1), xb), fmaxf(float(ix), xa)), 0.f);
                    OH[k * NS + i] = fmaxf(__fsub_rn(fminf(float(iy + 1), yb), fmaxf(float(iy), ya)), 0.f);
                    OD[k * NS + i] = fmaxf(__fsub_rn(fminf(float(iz + 1), zb), fmaxf(float(iz), za)), 0.f);
                }
            }
        }
    };
    auto term = [&](float m, float vol) -> float {
        if (POW2) return __fmul_rn(m, vol);
        return (m != 0.f && vol > 0.f) ? __fmul_rn(m, __fdiv_rn(vol, fp.total_area)) : 0.f;
    };
    const int lx = tid & (G3_W - 1), ly = tid / G3_W;
    const int X = x0 + lx, Y = y0 + ly;
    const bool inside = X < W && Y < H;
    // The wrapped-ascending x order (rot_window) is the natural order
    // kx = -RN..RN+1 rotated left by rx, so the terms are computed at fixed
    // shared-memory offsets and rotated in registers before they are added.
    const int rx = window_rotation(X, RN, W);
    // One output plane Z, its source planes in wrapped-ascending z order.
    auto single = [&](int Z) {
        float acc = 0.f;
        for (int jz = 0; jz < NW; ++jz) {
            const int kz = rot_window(jz, Z, RN, D);
            const float* P = slot(Z + kz);
            const float* OW = P;
            const float* OHk = P + NW * NS;
            const float* ODk = P + 2 * NW * NS + (kz + RN) * NS;
            const float* Mm = P + 3 * NW * NS;
#pragma unroll
            for (int jy = 0; jy < NW; ++jy) {
                const int ky = rot_window(jy, Y, RN, H);
                const int base = (ly + ky + RN) * SW + lx;  // source of kx = -RN
                const float* OHr = OHk + (ky + RN) * NS + base;
                float t[NW];
#pragma unroll
                for (int i = 0; i < NW; ++i)
                    t[i] = term(Mm[base + i], __fmul_rn(__fmul_rn(OW[i * NS + base + i], OHr[i]), ODk[base + i]));
                rotate_left<NW>(t, rx);
#pragma unroll
                for (int i = 0; i < NW; ++i) acc = __fadd_rn(acc, t[i]);
            }
        }
        out[(size_t(Z) * H + Y) * W + X] = acc;
    };
    // Output planes Z and Z+1 whose z windows do not wrap: source planes
    // Z-RN .. Z+RN+2 in ascending order, the first for Z only, the last for
    // Z+1 only; each destination adds its terms in the same order as single().
    auto pair = [&](int Z) {
        float acc0 = 0.f, acc1 = 0.f;
#pragma unroll
        for (int r = 0; r <= NW; ++r) {
            const float* P = slot(Z - RN + r);
            const float* OW = P;
            const float* OHk = P + NW * NS;
            const float* OD0 = P + 2 * NW * NS + r * NS;        // kz = r - RN for plane Z
            const float* OD1 = P + 2 * NW * NS + (r - 1) * NS;  // kz = r - RN - 1 for plane Z+1
            const float* Mm = P + 3 * NW * NS;
#pragma unroll
            for (int jy = 0; jy < NW; ++jy) {
                const int ky = rot_window(jy, Y, RN, H);
                const int base = (ly + ky + RN) * SW + lx;
                const float* OHr = OHk + (ky + RN) * NS + base;
                float t0[NW], t1[NW];
#pragma unroll
                for (int i = 0; i < NW; ++i) {
                    const float m = Mm[base + i];
                    const float wh = __fmul_rn(OW[i * NS + base + i], OHr[i]);
                    if (r < NW) t0[i] = term(m, __fmul_rn(wh, OD0[base + i]));
                    if (r > 0) t1[i] = term(m, __fmul_rn(wh, OD1[base + i]));
                }
                if (r < NW) {
                    rotate_left<NW>(t0, rx);
#pragma unroll
                    for (int i = 0; i < NW; ++i) acc0 = __fadd_rn(acc0, t0[i]);
                }
                if (r > 0) {
                    rotate_left<NW>(t1, rx);
#pragma unroll
                    for (int i = 0; i < NW; ++i) acc1 = __fadd_rn(acc1, t1[i]);
                }
            }
        }
        out[(size_t(Z) * H + Y) * W + X] = acc0;
        out[(size_t(Z + 1) * H + Y) * W + X] = acc1;
    };
    if constexpr (!G3_PAIRS) {
        float raw[4][NSP];
        for (int gz = z0 - RN; gz <= z0 + RN; ++gz) {
            fetch(gz, raw);
            store(gz, raw);
        }
        fetch(z0 + RN + 1, raw);
        for (int zz = 0; zz < nz; ++zz) {
            const int Z = z0 + zz;
            store(Z + RN + 1, raw);
            __syncthreads();
            if (zz + 1 < nz) fetch(Z + RN + 2, raw);
            if (inside) single(Z);
            __syncthreads();
        }
    } else {
        float ra[4][NSP], rb[4][NSP];
        for (int gz = z0 - RN; gz <= z0 + RN; ++gz) {
            fetch(gz, ra);
            store(gz, ra);
        }
        fetch(z0 + RN + 1, ra);
        if (nz > 1) fetch(z0 + RN + 2, rb);
        for (int zz = 0; zz < nz; zz += 2) {
            const int Z = z0 + zz;
            const bool two = zz + 1 < nz;
            store(Z + RN + 1, ra);
            if (two) store(Z + RN + 2, rb);
            __syncthreads();
            if (zz + 2 < nz) fetch(Z + RN + 3, ra);
            if (zz + 3 < nz) fetch(Z + RN + 4, rb);
            if (inside) {
                if (!two) {
                    single(Z);
                } else if (Z - RN >= 0 && Z + RN + 2 < D) {
                    pair(Z);
                } else {
                    single(Z);
                    single(Z + 1);
                }
            }
            __syncthreads();
        }
    }
}

inline size_t gather3d_dyn_smem() {
    const size_t a = March3<1>::bytes, b = sizeof(float) * 4 * G3_CELLS;
    return a > b ? a : b;
}

// Grid: (x tiles, y tiles, channels * z chunks of G3_NZ planes).
template <bool POW2>
__global__ void __launch_bounds__(256) gather_3d(const float* __restrict__ DX, const float* __restrict__ DY,
                                                 const float* __restrict__ DZ, const float* __restrict__ A,
                                                 float* __restrict__ Anext, int C, int W, int H, int D, FlowParams fp,
                                                 const int* __restrict__ dmax_slot) {
    dep_enter();
    extern __shared__ __align__(16) float sm[];
    const int nchunk = (D + G3_NZ - 1) / G3_NZ;
    const int c = blockIdx.z / nchunk;
    const int z0 = (blockIdx.z - c * nchunk) * G3_NZ;
    const int nz = min(G3_NZ, D - z0);
    const size_t N = size_t(W) * H * D, off = size_t(c) * N;
    const int RN = window_from_dmax(*dmax_slot, fp, max(max(W, H), D));
    const bool fast = RN <= G3_RNMAX && 2 * RN + 2 <= W && 2 * RN + 2 <= H && 2 * RN + 2 <= D && !fp.point_mode;
    const float *dx = DX + off, *dy = DY + off, *dz = DZ + off, *ms = A + off;  // ms: the state (source masses)
    float* o = Anext + off;
    if (fast && RN == 0) {
        gather3d_march<0, POW2>(sm, dx, dy, dz, ms, o, W, H, D, z0, nz, fp);
        return;
    }
    if (fast && RN == 1) {
        gather3d_march<1, POW2>(sm, dx, dy, dz, ms, o, W, H, D, z0, nz, fp);
        return;
    }
    for (int Z = z0; Z < z0 + nz; ++Z) {
        if (fast) {
            gather3d_plane<2, POW2>(sm, dx, dy, dz, ms, o, W, H, D, Z, fp);
            __syncthreads();
        } else {
            const int X = blockIdx.x * G3_W + (threadIdx.x & (G3_W - 1)), Y = blockIdx.y * G3_H + (threadIdx.x / G3_W);
            if (X < W && Y < H)
                o[(size_t(Z) * H + Y) * W + X] = gather3d_generic<POW2>(dx, dy, dz, ms, W, H, D, X, Y, Z, RN + 1, fp);
        }
    }
}

size_t gather3d_smem_bytes() { return gather3d_dyn_smem(); }

void launch_flow_3d(const float* A, const float* U, float* DX, float* DY, float* DZ, int C, int W, int H, int D,
                    const FlowParams& fp, int* dmax_slot, int* status, cudaStream_t st) {
    const int nz = flow3d_nz(C);
    dim3 grid((W + F3_W - 1) / F3_W, (H + F3_H - 1) / F3_H, (D + nz - 1) / nz);
    const size_t smem = flow3d_smem_bytes(C, nz);
    if (nz == 4) launch_dep(flow_3d<4>, grid, 256, smem, st, A, U, DX, DY, DZ, C, W, H, D, fp, dmax_slot, status);
    else launch_dep(flow_3d<2>, grid, 256, smem, st, A, U, DX, DY, DZ, C, W, H, D, fp, dmax_slot, status);
}

void launch_gather_3d(const float* DX, const float* DY, const float* DZ, const float* A, float* Anext, int C, int W,
                      int H, int D, const FlowParams& fp, const int* dmax_slot, cudaStream_t st) {
    dim3 grid((W + G3_W - 1) / G3_W, (H + G3_H - 1) / G3_H, C * ((D + G3_NZ - 1) / G3_NZ));
    if (fp.area_pow2)
        launch_dep(gather_3d<true>, grid, 256, gather3d_smem_bytes(), st, DX, DY, DZ, A, Anext, C, W, H, D, fp, dmax_slot);
    else
        launch_dep(gather_3d<false>, grid, 256, gather3d_smem_bytes(), st, DX, DY, DZ, A, Anext, C, W, H, D, fp, dmax_slot);
}

void transport_3d_set_attributes() {
    auto set = [](const void* f, size_t bytes) {
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    };
    const int c4 = int((F3_SMEM_MAX / (sizeof(float) * f3_rc(4)) - 1) / 2);  // most channels with four planes
    set((const void*)flow_3d<4>, flow3d_smem_bytes(c4, 4));
    set((const void*)flow_3d<2>, flow3d_smem_bytes(flow3d_max_channels(), 2));
    set((const void*)gather_3d<true>, gather3d_smem_bytes());
    set((const void*)gather_3d<false>, gather3d_smem_bytes());
}

}  // namespace flp
