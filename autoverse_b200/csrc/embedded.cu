// Parameter-embedded Flow Lenia on the device: the reference's
// EmbeddedPropagator (src/compute/embedded_propagator.rs:222-339), where every
// cell carries its own growth and flow parameters (CellParams: mu, sigma,
// weight, beta_a, n; schema/embedding.rs:20-31) and those parameters travel
// with the mass.
//
// A step is three stages:
//   * emb_conv_growth — for each target channel, the direct torus correlation
//     of every kernel aimed at it, in kernel order, with the growth evaluated
//     per cell from that channel's parameter grid (direct_convolution.rs:
//     133-177, embedded_propagator.rs:235-247).  For kernels of radius >= 8
//     on grids the FFT passes serve, the correlation sums come instead from
//     the engine's FFT convolution (rows R2C, columns with the spectrum
//     product, raw inverse rows: one plane per kernel; the stencils are
//     symmetric, so convolution and correlation agree) and emb_growth applies
//     the per-cell growth; the sums then differ from the direct ones by f32
//     rounding only;
//   * emb_flow — channel sum, Sobel gradients of the sum and of each
//     affinity, alpha from the cell's own beta_a and n, the flow and the
//     destinations (embedded_propagator.rs:249-300, 353-372); it also
//     publishes each channel's largest flow magnitude (param_advection.rs:
//     303-309) and the largest displacement of a mass-carrying cell;
//   * emb_gather — with embedding enabled, the reference's own gather: each
//     destination visits the (2R+1)^2 wrapped offsets in dy-major order, sums
//     the mass each source's square delivers and mixes the sources'
//     parameters (softmax or linear, embedding.rs:64-166); with embedding
//     disabled, the plain gather_2d (advect_mass_into, bit-exact) and the
//     parameters do not change.
//
// The parameter grids are double-buffered like the reference's propagator,
// which swaps its own buffer with the state's each step
// (embedded_propagator.rs:335-336): a destination that receives no mass keeps
// whatever the other buffer held.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "device_mem.h"
#include "common.cuh"
#include "flowlenia_cuda.h"
#include "kernels.h"
#include "schema.h"

namespace flp {

extern thread_local std::string g_last_error;

namespace {

constexpr int NPAR = 5;                                                  // CellParams fields
constexpr float CELL_DEFAULT[NPAR] = {0.15f, 0.015f, 1.0f, 1.0f, 2.0f};  // CellParams::default
constexpr int EMB_MAX_RADIUS = 64;
constexpr int EMB_GRAPH_STEPS = 16;  // even: a replay returns both buffers to their parity
constexpr int EC_TW = 32, EC_TH = 16;  // direct convolution tile (32x8 threads, 2 rows each)
constexpr int EC_RPT = EC_TH / 8;
constexpr int EG_T = 16;               // gather tile (16x16 threads, one destination each)
constexpr int EG_RSM = 8;              // windows up to this R stage their sources in shared memory
constexpr int EMB_FFT_MIN_RADIUS = 8;  // the FFT convolution serves kernels at least this wide

struct EKern {
    int src, tgt, size, tap_off;  // taps: the nonzero taps in ky-major order
    int n_taps;
};

void cke(cudaError_t e, const char* what) { throw_cuda(e, what); }

struct UnsupportedError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// input tile with halo, then the kernel's nonzero taps: value and packed (ky, kx)
size_t conv_smem(int rmax) {
    return sizeof(float) * (size_t(EC_TH + 2 * rmax) * (EC_TW + 2 * rmax) + 2 * size_t(2 * rmax + 1) * (2 * rmax + 1));
}
constexpr int EG_CMAX = 16;  // contributions per destination kept in shared memory
constexpr int EG_STAGE = (3 + NPAR) * (EG_T + 2 * EG_RSM) * (EG_T + 2 * EG_RSM);  // staged source planes
// staged sources, then per thread EG_CMAX contributions (f32) and their window offsets (u8)
size_t gather_smem() { return sizeof(float) * (EG_STAGE + EG_CMAX * 256) + EG_CMAX * 256; }

// ---------------------------------------------------------------- kernels --

// Direct correlation of each kernel aimed at channel blockIdx.z (reference
// orientation: output (x, y) reads input (x + kx - r, y + ky - r) times
// k[ky][kx]), summed tap by tap in ky-major order over the nonzero taps (the
// reference skips zero taps, direct_convolution.rs:149-151) without
// contraction, then the growth with the cell's own mu, sigma and weight,
// accumulated over the kernels in kernel order.  Block 32x8, EC_RPT rows per
// thread.  slots[0 .. nslots) are cleared for the flow pass that follows.
// taps: per kernel n_taps values, then n_taps packed (ky << 16 | kx).
__global__ void __launch_bounds__(256) emb_conv_growth(const float* __restrict__ A, float* __restrict__ U,
                                                       const float* __restrict__ P, const EKern* __restrict__ ek,
                                                       int K, const float* __restrict__ taps, int W, int H, int rmax,
                                                       int* slots, int nslots) {
    dep_enter();
    extern __shared__ float sm[];
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    const int c = blockIdx.z;
    const int x0 = blockIdx.x * EC_TW, y0 = blockIdx.y * EC_TH;
    const size_t N = size_t(W) * H;
    if (slots && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0)
        for (int i = tid; i < nslots; i += 256) slots[i] = 0;
    const int Pmax = EC_TW + 2 * rmax;
    float* tile = sm;                                       // (EC_TH + 2r) x (EC_TW + 2r)
    float* tval = sm + size_t(EC_TH + 2 * rmax) * Pmax;     // nonzero tap values
    int* toff = reinterpret_cast<int*>(tval + (2 * rmax + 1) * (2 * rmax + 1));  // their tile offsets
    // the target channel's growth parameters of this thread's cells
    float mu[EC_RPT], sig[EC_RPT], wgt[EC_RPT], u[EC_RPT];
#pragma unroll
    for (int i = 0; i < EC_RPT; ++i) {
        const int x = min(x0 + tx, W - 1), y = min(y0 + ty + 8 * i, H - 1);
        const size_t idx = size_t(y) * W + x;
        mu[i] = P[(size_t(c) * NPAR + 0) * N + idx];
        sig[i] = P[(size_t(c) * NPAR + 1) * N + idx];
        wgt[i] = P[(size_t(c) * NPAR + 2) * N + idx];
        u[i] = 0.f;
    }
    int loaded_src = -1, loaded_r = -1;
    for (int k = 0; k < K; ++k) {
        const EKern d = ek[k];
        if (d.tgt != c) continue;
        const int r = d.size / 2, P2 = EC_TW + 2 * r, nt = d.n_taps;
        __syncthreads();
        for (int i = tid; i < nt; i += 256) {
            tval[i] = taps[d.tap_off + i];
            const int packed = __float_as_int(taps[d.tap_off + nt + i]);
            toff[i] = (packed >> 16) * P2 + (packed & 0xFFFF);
        }
        if (d.src != loaded_src || r != loaded_r) {
            const float* a = A + size_t(d.src) * N;
            const int rows = EC_TH + 2 * r;
            for (int i = tid; i < rows * P2; i += 256) {
                const int ly = i / P2, lx = i - ly * P2;
                tile[i] = a[size_t(wrap_coord(y0 - r + ly, H)) * W + wrap_coord(x0 - r + lx, W)];
            }
            loaded_src = d.src;
            loaded_r = r;
        }
        __syncthreads();
        float acc[EC_RPT];
#pragma unroll
        for (int i = 0; i < EC_RPT; ++i) acc[i] = 0.f;
        const float* base = tile + ty * P2 + tx;
#pragma unroll 4
        for (int j = 0; j < nt; ++j) {
            const float t = tval[j];
            const float* b = base + toff[j];
#pragma unroll
            for (int i = 0; i < EC_RPT; ++i) acc[i] = __fadd_rn(acc[i], __fmul_rn(b[(8 * i) * P2], t));
        }
#pragma unroll
        for (int i = 0; i < EC_RPT; ++i) {
            // G(u; mu, sigma) = 2 exp(-(u - mu)^2 / (2 sigma^2)) - 1, times the cell's weight
            const float diff = __fsub_rn(acc[i], mu[i]);
            const float s2 = __fmul_rn(__fmul_rn(2.0f, sig[i]), sig[i]);
            const float g = __fsub_rn(__fmul_rn(2.0f, expf(__fdiv_rn(__fmul_rn(-diff, diff), s2))), 1.0f);
            u[i] = __fadd_rn(u[i], __fmul_rn(wgt[i], g));
        }
    }
#pragma unroll
    for (int i = 0; i < EC_RPT; ++i) {
        const int y = y0 + ty + 8 * i, x = x0 + tx;
        if (x < W && y < H) U[size_t(c) * N + size_t(y) * W + x] = u[i];
    }
}

// Growth of the FFT path: conv holds one plane per kernel (the correlation
// sums); U[c] = sum over the kernels aimed at c, in kernel order, of the
// cell's weight times G(conv; mu, sigma) of the cell.  One thread per cell of
// channel blockIdx.y.  slots[0 .. nslots) are cleared for the flow pass.
__global__ void __launch_bounds__(256) emb_growth(const float* __restrict__ conv, float* __restrict__ U,
                                                  const float* __restrict__ P, const EKern* __restrict__ ek, int K,
                                                  int W, int H, int* slots, int nslots) {
    dep_enter();
    const size_t N = size_t(W) * H;
    const int c = blockIdx.y;
    if (slots && blockIdx.x == 0 && blockIdx.y == 0)
        for (int i = threadIdx.x; i < nslots; i += 256) slots[i] = 0;
    const size_t i = size_t(blockIdx.x) * 256 + threadIdx.x;
    if (i >= N) return;
    const float mu = P[(size_t(c) * NPAR + 0) * N + i];
    const float sig = P[(size_t(c) * NPAR + 1) * N + i];
    const float wgt = P[(size_t(c) * NPAR + 2) * N + i];
    const float s2 = __fmul_rn(__fmul_rn(2.0f, sig), sig);
    float u = 0.f;
    for (int k = 0; k < K; ++k) {
        if (ek[k].tgt != c) continue;
        const float diff = __fsub_rn(conv[size_t(k) * N + i], mu);
        const float g = __fsub_rn(__fmul_rn(2.0f, expf(__fdiv_rn(__fmul_rn(-diff, diff), s2))), 1.0f);
        u = __fadd_rn(u, __fmul_rn(wgt, g));
    }
    U[size_t(c) * N + i] = u;
}

// Channel sum at (x, y) in channel order.
__device__ __forceinline__ float chan_sum(const float* __restrict__ A, int C, size_t N, size_t idx) {
    float s = 0.f;
    for (int c = 0; c < C; ++c) s = __fadd_rn(s, A[size_t(c) * N + idx]);
    return s;
}

// One thread per cell (block 32x8).  Writes destinations DX/DY for every
// channel; slots[0] takes the largest |dest - x| of a mass-carrying cell,
// slots[1 + c] channel c's largest flow magnitude over all cells.
__global__ void __launch_bounds__(256) emb_flow(const float* __restrict__ A, const float* __restrict__ U,
                                                const float* __restrict__ P, float* __restrict__ DX,
                                                float* __restrict__ DY, int C, int W, int H, FlowParams fp,
                                                int* slots, int* status) {
    dep_enter();
    const int x = blockIdx.x * 32 + (threadIdx.x & 31), y = blockIdx.y * 8 + (threadIdx.x >> 5);
    const bool in = x < W && y < H;
    const size_t N = size_t(W) * H;
    const int xp = in ? (x + W - 1) % W : 0, xn = in ? (x + 1) % W : 0;
    const int yp = in ? (y + H - 1) % H : 0, yn = in ? (y + 1) % H : 0;
    const size_t rp = size_t(yp) * W, rc = size_t(in ? y : 0) * W, rn = size_t(yn) * W;
    const int xc = in ? x : 0;
    float gax = 0.f, gay = 0.f, msum = 0.f, dmax = 0.f;
    bool bad = false;
    if (in) {
        sobel2(chan_sum(A, C, N, rp + xp), chan_sum(A, C, N, rp + xc), chan_sum(A, C, N, rp + xn),
               chan_sum(A, C, N, rc + xp), chan_sum(A, C, N, rc + xn), chan_sum(A, C, N, rn + xp),
               chan_sum(A, C, N, rn + xc), chan_sum(A, C, N, rn + xn), gax, gay);
        msum = chan_sum(A, C, N, rc + xc);
    }
    const size_t idx = rc + xc;
    const int lane = threadIdx.x & 31;
    for (int c = 0; c < C; ++c) {
        float fmag = 0.f;
        if (in) {
            const float* u = U + size_t(c) * N;
            float gux, guy;
            sobel2(u[rp + xp], u[rp + xc], u[rp + xn], u[rc + xp], u[rc + xn], u[rn + xp], u[rn + xc], u[rn + xn],
                   gux, guy);
            const float beta = P[(size_t(c) * NPAR + 3) * N + idx], nexp = P[(size_t(c) * NPAR + 4) * N + idx];
            const float alpha = flow_alpha(msum, beta, nexp);
            const float oma = __fsub_rn(1.0f, alpha);
            const float fx = __fsub_rn(__fmul_rn(oma, gux), __fmul_rn(alpha, gax));
            const float fy = __fsub_rn(__fmul_rn(oma, guy), __fmul_rn(alpha, gay));
            const float dx = __fadd_rn(float(x), __fmul_rn(fp.dt, fx));
            const float dy = __fadd_rn(float(y), __fmul_rn(fp.dt, fy));
            const float mass = A[size_t(c) * N + idx];
            bad |= !(isfinite(mass) && isfinite(dx) && isfinite(dy));
            if (fabsf(mass) >= 1e-10f) dmax = fmaxf(dmax, fmaxf(fabsf(dx - float(x)), fabsf(dy - float(y))));
            DX[size_t(c) * N + idx] = dx;
            DY[size_t(c) * N + idx] = dy;
            fmag = sqrtf(__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)));  // NaN is skipped like f32::max
        }
        for (int o = 16; o > 0; o >>= 1) fmag = fmaxf(fmag, __shfl_xor_sync(0xffffffffu, fmag, o));
        if (lane == 0 && fmag > 0.f) atomicMax(slots + 1 + c, __float_as_int(fmag));
    }
    if (status && __syncthreads_or(bad ? 1 : 0) && threadIdx.x == 0) atomicOr(status, STATUS_NONFINITE);
    for (int o = 16; o > 0; o >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if (lane == 0) {
        if (bad) dmax = INFINITY;
        if (dmax > 0.f) atomicMax(slots, __float_as_int(dmax));
    }
}

// compute_distribution_overlap (param_advection.rs:263-300): the source's
// square at (dfx, dfy) of half-side s against the cell [cx, cx+1) x [cy, cy+1).
// A power-of-two area divides exactly as a multiplication by its reciprocal.
__device__ __forceinline__ float emb_overlap(float dfx, float dfy, float s, float cx, float cy, float total_area,
                                             bool point, bool pow2, float inv_area) {
    const float cx1 = __fadd_rn(cx, 1.0f), cy1 = __fadd_rn(cy, 1.0f);
    if (point) return (cx <= dfx && dfx < cx1 && cy <= dfy && dfy < cy1) ? 1.0f : 0.0f;
    const float ox0 = fmaxf(__fsub_rn(dfx, s), cx), ox1 = fminf(__fadd_rn(dfx, s), cx1);
    const float ow = fmaxf(__fsub_rn(ox1, ox0), 0.f);
    // without x overlap the area is 0 (or NaN), which never contributes: skip the rest
    if (!(ow > 0.f)) return 0.f;
    const float oy0 = fmaxf(__fsub_rn(dfy, s), cy), oy1 = fminf(__fadd_rn(dfy, s), cy1);
    const float oh = fmaxf(__fsub_rn(oy1, oy0), 0.f);
    const float area = __fmul_rn(ow, oh);
    return pow2 ? __fmul_rn(area, inv_area) : __fdiv_rn(area, total_area);
}

// The gather of advect_mass_and_params_into for channel blockIdx.z, one
// destination per thread.  R = ceil(max|F| dt + s) + 1 from the channel's
// largest flow magnitude; the sources of the tile's window are staged in
// shared memory when R <= EG_RSM.  Mass: the contributions m * overlap of
// the sources (|m| >= 1e-10, overlap > 0) summed in offset order.
// Parameters: written only when mass arrives (total > 1e-10); one source
// passes its parameters on, more are mixed: linear (w = m_i / total) or
// softmax (w_i = exp((m_i - max m) / T) / sum_j exp(...)), the weighted sums
// accumulated in offset order, as mix_linear / mix_softmax do.
__global__ void __launch_bounds__(256) emb_gather(const float* __restrict__ A, const float* __restrict__ DX,
                                                  const float* __restrict__ DY, const float* __restrict__ P,
                                                  float* __restrict__ An, float* __restrict__ Pn, int W, int H,
                                                  FlowParams fp, int linear, float temperature,
                                                  const int* __restrict__ slots) {
    dep_enter();
    extern __shared__ float sm[];
    const int c = blockIdx.z;
    const size_t N = size_t(W) * H;
    const float* mass = A + size_t(c) * N;
    const float* dxp = DX + size_t(c) * N;
    const float* dyp = DY + size_t(c) * N;
    const float dt = fp.dt, s = fp.s;
    const float fm = __int_as_float(slots[1 + c]);
    const float rv = ceilf(__fadd_rn(__fmul_rn(fm, dt), s));
    // The reference's window: Rust `as i32` saturates (NaN -> 0); capped at
    // twice the larger side, far beyond any mass-conserving flow.
    const int cap = 2 * max(W, H);
    const int R_ref = 1 + (rv != rv ? 0 : (rv >= float(cap) ? cap : (rv <= -float(cap) ? -cap : int(rv))));
    // Only sources with |m| >= 1e-10 contribute, and such a source at offset o
    // reaches the destination only if |o| <= ceil(s + D) (D: the largest
    // |dest - x| of a mass-carrying cell, slots[0]; one more cell for the
    // nearest-cell mode).  Visiting that sub-window in the same dy-major order
    // gives the same contributions in the same order, unless the reference's
    // window wraps the torus (it can then visit a source twice): keep it there.
    int R = R_ref;
    if (2 * R_ref + 1 <= W && 2 * R_ref + 1 <= H) {
        const float rd = ceilf(__fadd_rn(__fadd_rn(__int_as_float(slots[0]), fp.pos_eps), s));
        const int Rd = (rd < float(R_ref) ? int(rd) : R_ref) + (fp.point_mode ? 1 : 0);
        R = min(R_ref, max(Rd, 0));
    }
    const int tx = threadIdx.x & (EG_T - 1), ty = threadIdx.x / EG_T;
    const int x0 = blockIdx.x * EG_T, y0 = blockIdx.y * EG_T;
    const int dest_x = x0 + tx, dest_y = y0 + ty;
    const bool staged = R >= 0 && R <= EG_RSM;
    const int SW = EG_T + 2 * max(R, 0);
    // staged planes over the tile's window: mass, destinations, the 5 parameters
    float* sm_m = sm;
    float* sm_x = sm + SW * SW;
    float* sm_y = sm + 2 * SW * SW;
    float* sm_p = sm + 3 * SW * SW;
    const float* Pc = P + size_t(c) * NPAR * N;
    if (staged) {
        for (int i = threadIdx.x; i < SW * SW; i += 256) {
            const int ly = i / SW, lx = i - ly * SW;
            const size_t src = size_t(wrap_coord(y0 - R + ly, H)) * W + wrap_coord(x0 - R + lx, W);
            sm_m[i] = mass[src];
            sm_x[i] = dxp[src];
            sm_y[i] = dyp[src];
#pragma unroll
            for (int f = 0; f < NPAR; ++f) sm_p[f * SW * SW + i] = Pc[size_t(f) * N + src];
        }
        __syncthreads();
    }
    // field f of a source: `src` is its window index when staged, else its cell index
    auto param = [&](int f, size_t src) { return staged ? sm_p[f * SW * SW + src] : Pc[size_t(f) * N + src]; };
    if (dest_x >= W || dest_y >= H) return;
    const float total_area = fp.total_area;  // (2s)*(2s) in f32 (param_advection.rs:290)
    const bool point = !(total_area > 1e-10f);
    const bool pow2 = fp.area_pow2 != 0;
    const float cx = float(dest_x), cy = float(dest_y);
    const int side = 2 * R + 1;
    // window offset (dy, dx): whether the source contributes (|m| >= 1e-10 and
    // a positive overlap), its contribution m * overlap and its index
    auto contrib = [&](int dy, int dx, float& mc, size_t& src) -> bool {
        float m, fx, fy;
        if (staged) {
            const int li = (ty + R + dy) * SW + (tx + R + dx);
            src = size_t(li);
            m = sm_m[li];
            fx = sm_x[li];
            fy = sm_y[li];
        } else {
            src = size_t(wrap_coord(dest_y + dy, H)) * W + wrap_coord(dest_x + dx, W);
            m = mass[src];
            fx = dxp[src];
            fy = dyp[src];
        }
        if (fabsf(m) < 1e-10f) return false;
        const float ov = emb_overlap(fx, fy, s, cx, cy, total_area, point, pow2, fp.inv_area);
        if (!(ov > 0.f)) return false;
        mc = __fmul_rn(m, ov);
        return true;
    };
    // pass 1: mass, contribution count, largest contribution, first source; the
    // first EG_CMAX contributions and their window offsets stay in shared memory
    float* cmem = sm + EG_STAGE;                                                  // [e * 256 + thread]
    unsigned char* cidx = reinterpret_cast<unsigned char*>(cmem + EG_CMAX * 256);  // [e * 256 + thread]
    const int tid = threadIdx.x;
    const bool keep = side * side <= 256;  // offsets fit a byte
    float total = 0.f, maxm = -INFINITY;
    int n = 0;
    size_t first = 0;
    for (int dy = -R; dy <= R; ++dy)
        for (int dx = -R; dx <= R; ++dx) {
            float mc;
            size_t src;
            if (!contrib(dy, dx, mc, src)) continue;
            total = __fadd_rn(total, mc);
            maxm = fmaxf(maxm, mc);
            if (n == 0) first = src;
            if (keep && n < EG_CMAX) {
                cmem[n * 256 + tid] = mc;
                cidx[n * 256 + tid] = static_cast<unsigned char>((dy + R) * side + (dx + R));
            }
            ++n;
        }
    const size_t dest = size_t(dest_y) * W + dest_x;
    An[size_t(c) * N + dest] = total;
    if (!(n > 0 && total > 1e-10f)) return;  // the destination keeps the other buffer's parameters
    float out[NPAR];
    if (n == 1) {
#pragma unroll
        for (int f = 0; f < NPAR; ++f) out[f] = param(f, first);
    } else {
#pragma unroll
        for (int f = 0; f < NPAR; ++f) out[f] = 0.f;
        auto accumulate = [&](size_t src, float w) {
#pragma unroll
            for (int f = 0; f < NPAR; ++f)
                out[f] = __fadd_rn(out[f], __fmul_rn(param(f, src), w));
        };
        if (keep && n <= EG_CMAX) {
            // the contributions from shared memory, in offset order
            auto src_of = [&](int e) -> size_t {
                const int j = cidx[e * 256 + tid];
                const int dy = j / side - R, dx = j % side - R;
                if (staged) return size_t((ty + R + dy) * SW + (tx + R + dx));
                return size_t(wrap_coord(dest_y + dy, H)) * W + wrap_coord(dest_x + dx, W);
            };
            if (linear) {
                // mix_linear: w = m_i / total (total > 1e-10 here, so never the default)
                for (int e = 0; e < n; ++e) accumulate(src_of(e), __fdiv_rn(cmem[e * 256 + tid], total));
            } else {
                // mix_softmax: the weights once, kept in place of the contributions
                float wsum = 0.f;
                for (int e = 0; e < n; ++e) {
                    const float w = expf(__fdiv_rn(__fsub_rn(cmem[e * 256 + tid], maxm), temperature));
                    cmem[e * 256 + tid] = w;
                    wsum = __fadd_rn(wsum, w);
                }
                if (wsum > 0.f) {
                    for (int e = 0; e < n; ++e) accumulate(src_of(e), __fdiv_rn(cmem[e * 256 + tid], wsum));
                } else {
                    const float uni = __fdiv_rn(1.0f, float(n));
                    for (int e = 0; e < n; ++e) accumulate(src_of(e), uni);
                }
            }
        } else {
            // more contributions than kept: visit the window again in offset order
            auto for_each = [&](auto&& fn) {
                for (int dy = -R; dy <= R; ++dy)
                    for (int dx = -R; dx <= R; ++dx) {
                        float mc;
                        size_t src;
                        if (contrib(dy, dx, mc, src)) fn(mc, src);
                    }
            };
            if (linear) {
                for_each([&](float mc, size_t src) { accumulate(src, __fdiv_rn(mc, total)); });
            } else {
                float wsum = 0.f;
                for_each([&](float mc, size_t) {
                    wsum = __fadd_rn(wsum, expf(__fdiv_rn(__fsub_rn(mc, maxm), temperature)));
                });
                if (wsum > 0.f) {
                    for_each([&](float mc, size_t src) {
                        accumulate(src, __fdiv_rn(expf(__fdiv_rn(__fsub_rn(mc, maxm), temperature)), wsum));
                    });
                } else {
                    const float uni = __fdiv_rn(1.0f, float(n));
                    for_each([&](float, size_t src) { accumulate(src, uni); });
                }
            }
        }
    }
#pragma unroll
    for (int f = 0; f < NPAR; ++f) Pn[(size_t(c) * NPAR + f) * N + dest] = out[f];
}

std::once_flag g_eattr_once;

}  // namespace
}  // namespace flp

using namespace flp;

struct flp_embedded {
    SimulationConfig cfg;
    int W = 0, H = 0, C = 0, K = 0;
    size_t N = 0;
    FlowParams fp{};
    bool enabled = false, linear = false;
    float temperature = 1.0f;
    int rmax = 0;
    cudaStream_t st = nullptr;
    float* A[2] = {nullptr, nullptr};
    float* P[2] = {nullptr, nullptr};  // C x NPAR x N, field planes
    int cur = 0, pcur = 0;
    float *U = nullptr, *DX = nullptr, *DY = nullptr;
    int* d_slots = nullptr;  // [0] displacement bound, [1 + c] flow magnitude of channel c
    int* d_status = nullptr;
    EKern* d_ek = nullptr;
    float* d_taps = nullptr;
    double2* d_partial = nullptr;
    int np = 0;
    double* d_mass = nullptr;
    // FFT convolution (kernels of radius >= EMB_FFT_MIN_RADIUS on FFT grids)
    bool use_fft = false;
    FftGeom geom;
    float2 *d_tw = nullptr, *d_S = nullptr, *d_T = nullptr, *d_KH = nullptr;
    int *d_srcs = nullptr, *d_kslot = nullptr;
    int nsrc = 0;
    float* d_conv = nullptr;  // K planes of correlation sums
    std::vector<float> defaults;  // EmbeddedState::from_seed's CellParams
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    float time = 0.f;
    uint64_t step = 0;

    // profiling: events recorded after each of the three kernels when set
    cudaEvent_t* stage_ev = nullptr;
    void mark(int i) {
        if (stage_ev) cke(cudaEventRecord(stage_ev[i], st), "event");
    }

    void enqueue_step() {
        const float* a = A[cur];
        float* an = A[cur ^ 1];
        const float* p = P[pcur];
        mark(0);
        if (use_fft) {
            launch_fft_r2c(a, d_S, d_srcs, nsrc, W, H, geom, nullptr, 0, st);
            launch_fft_cols_conv(d_S, d_KH, d_T, d_kslot, nsrc, K, 1, W, H, geom, st);
            launch_fft_c2r_raw(d_T, d_conv, nullptr, K, W, H, 1.f, false, geom, st);
            launch_dep(emb_growth, dim3(unsigned((N + 255) / 256), C), dim3(256), size_t(0), st, (const float*)d_conv,
                       U, p, (const EKern*)d_ek, K, W, H, d_slots, 1 + C);
        } else {
            launch_dep(emb_conv_growth, dim3((W + EC_TW - 1) / EC_TW, (H + EC_TH - 1) / EC_TH, C), dim3(256),
                       conv_smem(rmax), st, a, U, p, (const EKern*)d_ek, K, (const float*)d_taps, W, H, rmax,
                       d_slots, 1 + C);
        }
        mark(1);
        launch_dep(emb_flow, dim3((W + 31) / 32, (H + 7) / 8), dim3(256), size_t(0), st, a, (const float*)U, p, DX,
                   DY, C, W, H, fp, d_slots, d_status);
        mark(2);
        if (enabled) {
            launch_dep(emb_gather, dim3((W + EG_T - 1) / EG_T, (H + EG_T - 1) / EG_T, C), dim3(256), gather_smem(),
                       st, a, (const float*)DX, (const float*)DY, p, an, P[pcur ^ 1], W, H, fp, linear ? 1 : 0,
                       temperature, (const int*)d_slots);
            pcur ^= 1;
        } else {
            launch_gather_2d(DX, DY, a, an, C, W, H, fp, d_slots, 1, st);
        }
        mark(3);
        cke(cudaGetLastError(), "embedded step launch");
        cur ^= 1;
    }

    void advance(uint64_t n) {
        for (uint64_t i = 0; i < n; ++i) time += cfg.dt;  // f32 accumulation, embedded_propagator.rs:337
        step += n;
    }

    void build_graph() {
        const int c0 = cur, p0 = pcur;
        cudaGraph_t g = nullptr;
        cke(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
        try {
            for (int i = 0; i < EMB_GRAPH_STEPS; ++i) enqueue_step();
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            cur = c0;
            pcur = p0;
            throw;
        }
        cke(cudaStreamEndCapture(st, &g), "capture");
        cur = c0;
        pcur = p0;
        cudaGraphExec_t ge = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        cke(e, "graph instantiate");
        graph[c0][p0] = ge;
    }

    void run(uint64_t n) {
        while (n >= uint64_t(EMB_GRAPH_STEPS)) {
            if (!graph[cur][pcur]) build_graph();
            cke(cudaGraphLaunch(graph[cur][pcur], st), "graph launch");
            advance(EMB_GRAPH_STEPS);
            n -= EMB_GRAPH_STEPS;
        }
        for (uint64_t i = 0; i < n; ++i) {
            enqueue_step();
            advance(1);
        }
    }

    // AoS host grids [c][cell][field] <-> device field planes
    void upload_params(const float* aos) {
        std::vector<float> soa(size_t(C) * NPAR * N);
        for (int c = 0; c < C; ++c)
            for (size_t i = 0; i < N; ++i)
                for (int f = 0; f < NPAR; ++f) soa[(size_t(c) * NPAR + f) * N + i] = aos[(size_t(c) * N + i) * NPAR + f];
        cke(cudaMemcpyAsync(P[pcur], soa.data(), soa.size() * sizeof(float), cudaMemcpyHostToDevice, st), "upload");
        cke(cudaStreamSynchronize(st), "sync");
    }

    void fill_params(float* dst, const float* row) {
        std::vector<float> soa(size_t(C) * NPAR * N);
        for (int c = 0; c < C; ++c)
            for (int f = 0; f < NPAR; ++f) std::fill_n(soa.begin() + (size_t(c) * NPAR + f) * N, N, row[f]);
        cke(cudaMemcpy(dst, soa.data(), soa.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
    }

    void free_all() {
        for (auto& row : graph)
            for (auto& g : row)
                if (g) cudaGraphExecDestroy(g);
        void* ptrs[] = {A[0], A[1], P[0], P[1], U, DX, DY, d_slots, d_status, d_ek, d_taps, d_partial, d_mass,
                        d_tw, d_S, d_T, d_KH, d_srcs, d_kslot, d_conv};
        for (void* q : ptrs)
            if (q) flp::dfree(q);
        if (st) cudaStreamDestroy(st);
    }
};

namespace flp {
namespace {

template <class T>
T* ealloc(size_t n) {
    void* p = nullptr;
    cke(flp::dmalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "allocation");
    return static_cast<T*>(p);
}

void emb_create(flp_embedded* h, const char* json) {
    h->cfg = parse_config(json);
    const SimulationConfig& cfg = h->cfg;
    if (cfg.is_3d()) throw UnsupportedError("parameter embedding is 2D only (embedded_propagator.rs:43)");
    h->W = cfg.width;
    h->H = cfg.height;
    h->C = cfg.channels;
    h->K = int(cfg.kernels.size());
    h->N = size_t(h->W) * h->H;
    h->fp = flow_params_of(cfg);
    h->enabled = cfg.embedding_enabled;
    h->linear = cfg.embedding_linear;
    h->temperature = cfg.embedding_temperature;
    std::vector<EKern> ek;
    std::vector<float> taps;
    std::vector<KernelStencil> stencils;
    for (const KernelConfig& kc : cfg.kernels) {
        KernelStencil ks = build_kernel(kc, cfg.kernel_radius, 2);
        stencils.push_back(ks);
        if (ks.radius > EMB_MAX_RADIUS)
            throw UnsupportedError("embedded direct convolution supports kernel radii up to 64 cells");
        std::vector<float> vals, packed;
        for (int ky = 0; ky < ks.size; ++ky)
            for (int kx = 0; kx < ks.size; ++kx) {
                const float v = ks.data[size_t(ky) * ks.size + kx];
                if (v == 0.f) continue;
                vals.push_back(v);
                int pk = (ky << 16) | kx;
                float f;
                std::memcpy(&f, &pk, sizeof f);
                packed.push_back(f);
            }
        ek.push_back({kc.source_channel, kc.target_channel, ks.size, int(taps.size()), int(vals.size())});
        taps.insert(taps.end(), vals.begin(), vals.end());
        taps.insert(taps.end(), packed.begin(), packed.end());
        h->rmax = std::max(h->rmax, ks.radius);
    }
    std::call_once(g_eattr_once, [] {
        cudaFuncSetAttribute((const void*)emb_conv_growth, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(conv_smem(EMB_MAX_RADIUS)));
        cudaFuncSetAttribute((const void*)emb_gather, cudaFuncAttributeMaxDynamicSharedMemorySize, int(gather_smem()));
        transport_2d_set_attributes();
        fft2d_set_attributes(200 * 1024);
    });
    cke(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking), "stream");
    const size_t CN = size_t(h->C) * h->N;
    for (int i = 0; i < 2; ++i) {
        h->A[i] = ealloc<float>(CN);
        h->P[i] = ealloc<float>(CN * NPAR);
        cke(cudaMemset(h->A[i], 0, CN * sizeof(float)), "memset");
    }
    h->U = ealloc<float>(CN);
    h->DX = ealloc<float>(CN);
    h->DY = ealloc<float>(CN);
    h->d_slots = ealloc<int>(1 + h->C);
    h->d_status = ealloc<int>(1);
    cke(cudaMemset(h->d_slots, 0, sizeof(int) * (1 + h->C)), "memset");
    cke(cudaMemset(h->d_status, 0, sizeof(int)), "memset");
    h->d_ek = ealloc<EKern>(ek.size());
    h->d_taps = ealloc<float>(taps.size());
    if (!ek.empty()) cke(cudaMemcpy(h->d_ek, ek.data(), ek.size() * sizeof(EKern), cudaMemcpyHostToDevice), "upload");
    if (!taps.empty()) cke(cudaMemcpy(h->d_taps, taps.data(), taps.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
    // FFT convolution for wide kernels on grids the templated passes serve
    const int W = h->W, H = h->H;
    if (h->K > 0 && h->rmax >= EMB_FFT_MIN_RADIUS && W % 2 == 0 && fft_row_templated(W / 2) && fft_col_templated(H)) {
        FftGeom g;
        if (make_plan(W / 2, g.pm) && make_plan(H, g.ph)) {
            const int M = W / 2, Wc = M + 1;
            std::vector<float2> tw;
            auto twid = [&](int L, int count) {
                for (int t = 0; t < count; ++t) {
                    const double ang = -2.0 * M_PI * double(t) / double(L);
                    tw.push_back(make_float2(float(std::cos(ang)), float(std::sin(ang))));
                }
            };
            twid(M, M);
            twid(W, Wc);
            twid(H, H);
            h->d_tw = ealloc<float2>(tw.size());
            cke(cudaMemcpy(h->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice), "upload");
            g.twM = h->d_tw;
            g.twW = h->d_tw + M;
            g.twH = h->d_tw + M + Wc;
            h->geom = g;
            // the convolution's own passes: 4-warp CTAs, one column transform
            // per kernel (measured faster for a few kernels per world)
            h->geom.wpc_r2c = h->geom.wpc_cols = h->geom.wpc_c2r = 4;
            h->geom.share_cols = 0;
            std::vector<int> srcs, kslot(h->K);
            for (int k = 0; k < h->K; ++k) {
                auto it = std::find(srcs.begin(), srcs.end(), ek[k].src);
                if (it == srcs.end()) { kslot[k] = int(srcs.size()); srcs.push_back(ek[k].src); }
                else kslot[k] = int(it - srcs.begin());
            }
            h->nsrc = int(srcs.size());
            h->d_srcs = ealloc<int>(srcs.size());
            h->d_kslot = ealloc<int>(kslot.size());
            cke(cudaMemcpy(h->d_srcs, srcs.data(), srcs.size() * sizeof(int), cudaMemcpyHostToDevice), "upload");
            cke(cudaMemcpy(h->d_kslot, kslot.data(), kslot.size() * sizeof(int), cudaMemcpyHostToDevice), "upload");
            const size_t spec = size_t(Wc) * H;
            h->d_S = ealloc<float2>(spec * h->nsrc);
            h->d_T = ealloc<float2>(spec * h->K);
            h->d_KH = ealloc<float2>(spec * h->K);
            h->d_conv = ealloc<float>(size_t(h->K) * h->N);
            // kernel spectra of the wrap-padded stencils, scaled by 1/(W*H)
            std::vector<float> padded(size_t(h->K) * h->N);
            for (int k = 0; k < h->K; ++k) {
                const std::vector<float> pk = pad_kernel(stencils[k], W, H, 1);
                std::copy(pk.begin(), pk.end(), padded.begin() + size_t(k) * h->N);
            }
            DevScratch scratch;
            float* d_pad = scratch.add(ealloc<float>(padded.size()));
            float2* d_tmp = scratch.add(ealloc<float2>(spec * h->K));
            cke(cudaMemcpy(d_pad, padded.data(), padded.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
            launch_fft_r2c(d_pad, d_tmp, nullptr, h->K, W, H, g, nullptr, 0, h->st);
            launch_fft_cols(d_tmp, nullptr, h->d_KH, nullptr, h->K, W, H, g, 1, float(1.0 / (double(W) * double(H))),
                            h->st);
            cke(cudaGetLastError(), "kernel spectra");
            cke(cudaStreamSynchronize(h->st), "sync");
            h->use_fft = true;
        }
    }
    h->np = int(std::min<size_t>(1024, (CN + 255) / 256));
    h->d_partial = ealloc<double2>(h->np);
    h->d_mass = ealloc<double>(1);
    // EmbeddedState::from_seed's parameters (embedded_propagator.rs:51-58) in
    // the state's grids; CellParams::default in the propagator's own buffer
    // (embedded_propagator.rs:195-199)
    const KernelConfig* k0 = cfg.kernels.empty() ? nullptr : &cfg.kernels[0];
    h->defaults = {k0 ? k0->mu : 0.15f, k0 ? k0->sigma : 0.015f, k0 ? k0->weight : 1.0f, cfg.flow.beta_a, cfg.flow.n};
    h->fill_params(h->P[0], h->defaults.data());
    h->fill_params(h->P[1], CELL_DEFAULT);
}

int efail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace
}  // namespace flp

#define EMB_TRY(...)                                             \
    try {                                                        \
        __VA_ARGS__;                                             \
        return FLP_OK;                                           \
    } catch (const flp::ConfigError& e) {                        \
        return flp::efail(FLP_ERR_INVALID_CONFIG, e.what());     \
    } catch (const flp::UnsupportedError& e) {                   \
        return flp::efail(FLP_ERR_UNSUPPORTED, e.what());        \
    } catch (const std::invalid_argument& e) {                   \
        return flp::efail(FLP_ERR_INVALID_ARGUMENT, e.what());   \
    } catch (const std::bad_alloc&) {                            \
        return flp::efail(FLP_ERR_OOM, "host allocation failed"); \
    } catch (const flp::DeviceOom& e) {                          \
        return flp::efail(FLP_ERR_OOM, e.what());                \
    } catch (const std::exception& e) {                          \
        return flp::efail(FLP_ERR_CUDA, e.what());               \
    }

#define EMB_HANDLE(h) \
    if (!(h)) return flp::efail(FLP_ERR_INVALID_ARGUMENT, "null embedded handle");

extern "C" {

int flp_emb_create(const char* config_json, flp_embedded** out) {
    if (!config_json || !out) return efail(FLP_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    flp_embedded* h = new flp_embedded();
    try {
        emb_create(h, config_json);
    } catch (...) {
        h->free_all();
        delete h;
        EMB_TRY(throw)
    }
    *out = h;
    return FLP_OK;
}

int flp_emb_destroy(flp_embedded* h) {
    if (!h) return FLP_OK;
    cudaStreamSynchronize(h->st);
    h->free_all();
    delete h;
    return FLP_OK;
}

int flp_emb_state_from_seed(flp_embedded* h, const char* seed_json) {
    EMB_HANDLE(h);
    EMB_TRY({
        if (!seed_json) throw std::invalid_argument("null seed");
        const std::vector<float> g = generate_seed(seed_json, h->cfg);
        cke(cudaStreamSynchronize(h->st), "sync");
        cke(cudaMemcpy(h->A[h->cur], g.data(), g.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
        h->fill_params(h->P[h->pcur], h->defaults.data());
        h->time = 0.f;
        h->step = 0;
    })
}

int flp_emb_write_state(flp_embedded* h, const float* channels, size_t n, const float* params, size_t n_params,
                        float time, uint64_t step) {
    EMB_HANDLE(h);
    EMB_TRY({
        const size_t CN = size_t(h->C) * h->N;
        if (!channels || n != CN) throw std::invalid_argument("state size mismatch: expected " + std::to_string(CN));
        if (params && n_params != CN * 5) throw std::invalid_argument("parameter size mismatch: expected " + std::to_string(CN * 5));
        cke(cudaMemcpyAsync(h->A[h->cur], channels, CN * sizeof(float), cudaMemcpyHostToDevice, h->st), "upload");
        if (params) h->upload_params(params);
        cke(cudaStreamSynchronize(h->st), "sync");
        h->time = time;
        h->step = step;
    })
}

int flp_emb_read_state(flp_embedded* h, float* channels, size_t n, float* params, size_t n_params, float* time,
                       uint64_t* step) {
    EMB_HANDLE(h);
    EMB_TRY({
        const size_t CN = size_t(h->C) * h->N;
        if (channels && n != CN) throw std::invalid_argument("state size mismatch: expected " + std::to_string(CN));
        if (params && n_params != CN * 5) throw std::invalid_argument("parameter size mismatch: expected " + std::to_string(CN * 5));
        if (channels)
            cke(cudaMemcpyAsync(channels, h->A[h->cur], CN * sizeof(float), cudaMemcpyDeviceToHost, h->st), "download");
        std::vector<float> soa;
        if (params) {
            soa.resize(CN * 5);
            cke(cudaMemcpyAsync(soa.data(), h->P[h->pcur], soa.size() * sizeof(float), cudaMemcpyDeviceToHost, h->st),
                "download");
        }
        cke(cudaStreamSynchronize(h->st), "sync");
        if (params)
            for (int c = 0; c < h->C; ++c)
                for (size_t i = 0; i < h->N; ++i)
                    for (int f = 0; f < 5; ++f)
                        params[(size_t(c) * h->N + i) * 5 + f] = soa[(size_t(c) * 5 + f) * h->N + i];
        if (time) *time = h->time;
        if (step) *step = h->step;
    })
}

int flp_emb_step(flp_embedded* h) {
    EMB_HANDLE(h);
    EMB_TRY(h->run(1))
}

int flp_emb_run(flp_embedded* h, uint64_t n) {
    EMB_HANDLE(h);
    EMB_TRY(h->run(n))
}

int flp_emb_synchronize(flp_embedded* h) {
    EMB_HANDLE(h);
    try {
        cke(cudaStreamSynchronize(h->st), "sync");
        int status = 0;
        cke(cudaMemcpy(&status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost), "status");
        if (status) {
            cke(cudaMemset(h->d_status, 0, sizeof(int)), "status");
            return efail(FLP_ERR_NONFINITE, "non-finite mass in the state");
        }
    } catch (const std::exception& e) {
        return efail(FLP_ERR_CUDA, e.what());
    }
    return FLP_OK;
}

int flp_emb_total_mass(flp_embedded* h, double* out) {
    EMB_HANDLE(h);
    EMB_TRY({
        if (!out) throw std::invalid_argument("null output");
        launch_mass_fp64(h->A[h->cur], size_t(h->C) * h->N, h->d_partial, h->np, h->d_mass, h->st);
        cke(cudaGetLastError(), "mass");
        cke(cudaMemcpyAsync(out, h->d_mass, sizeof(double), cudaMemcpyDeviceToHost, h->st), "mass");
        cke(cudaStreamSynchronize(h->st), "sync");
    })
}

int flp_emb_profile_run(flp_embedded* h, uint64_t steps, float* step_ms, float* stage_ms) {
    EMB_HANDLE(h);
    EMB_TRY({
        cudaEvent_t ev[4];
        for (auto& e : ev) cke(cudaEventCreate(&e), "event");
        if (!stage_ms) {
            cke(cudaEventRecord(ev[0], h->st), "event");
            h->run(steps);
            cke(cudaEventRecord(ev[3], h->st), "event");
            cke(cudaEventSynchronize(ev[3]), "sync");
            float ms = 0.f;
            cke(cudaEventElapsedTime(&ms, ev[0], ev[3]), "elapsed");
            if (step_ms) *step_ms = ms;
        } else {
            // eager steps with events between the kernels: conv+growth, flow, gather
            float acc[3] = {0.f, 0.f, 0.f}, tot = 0.f;
            h->stage_ev = ev;
            try {
                for (uint64_t i = 0; i < steps; ++i) {
                    h->enqueue_step();
                    h->advance(1);
                    cke(cudaEventSynchronize(ev[3]), "sync");
                    for (int k = 0; k < 3; ++k) {
                        float ms = 0.f;
                        cke(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]), "elapsed");
                        acc[k] += ms;
                        tot += ms;
                    }
                }
            } catch (...) {
                h->stage_ev = nullptr;
                throw;
            }
            h->stage_ev = nullptr;
            for (int k = 0; k < 3; ++k) stage_ms[k] = acc[k];
            if (step_ms) *step_ms = tot;
        }
        for (auto& e : ev) cudaEventDestroy(e);
    })
}

void* flp_emb_stream(flp_embedded* h) { return h ? static_cast<void*>(h->st) : nullptr; }

}  // extern "C"
