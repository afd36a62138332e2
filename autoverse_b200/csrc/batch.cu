// Batched engine: many independent 2D worlds of uneven sizes, channel counts
// and parameters advanced together (the use the evolution search makes of the
// reference, one CpuPropagator per candidate: src/compute/evolution/search.rs:152-172,
// fitness.rs:26-88).
//
// All worlds share pooled buffers; a device descriptor per world gives its
// sizes, parameters and offsets.  A step is five persistent kernels, one per
// stage (row R2C, column convolution, row C2R + growth, flow, gather).  The
// CTAs of each kernel pull (world, tile) items from that stage's device work
// queue (an atomic counter over a precomputed item list, largest worlds
// first) and dispatch at run time into the same compile-time item functions
// the single-world kernels use, so a world gives bit-identical results in
// either engine.  Each stage resets the next stage's counter; run(n) replays
// a captured CUDA graph of the step loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "device_mem.h"
#include "fft_items.cuh"
#include "fft_warp.cuh"
#include "host_pool.h"
#include "flowlenia_cuda.h"
#include "kernels.h"
#include "schema.h"
#include "transport_items.cuh"

namespace flp {

extern thread_local std::string g_last_error;

namespace {

// Warps per CTA of the batched FFT passes and whether a column item serves
// every kernel of its source (one forward column transform per source) or a
// single kernel; compile-time choices, none of which changes a result bit.
#ifndef FLP_BATCH_WPC_R2C
#define FLP_BATCH_WPC_R2C 4
#endif
#ifndef FLP_BATCH_WPC_COLS
#define FLP_BATCH_WPC_COLS 4
#endif
#ifndef FLP_BATCH_WPC_C2R
#define FLP_BATCH_WPC_C2R 4
#endif
#ifndef FLP_BATCH_SHARE_COLS
#define FLP_BATCH_SHARE_COLS 1
#endif
constexpr int BATCH_WPC_R2C = FLP_BATCH_WPC_R2C;
constexpr int BATCH_WPC_COLS = FLP_BATCH_WPC_COLS;
constexpr int BATCH_WPC_C2R = FLP_BATCH_WPC_C2R;
constexpr bool BATCH_SHARE_COLS = FLP_BATCH_SHARE_COLS != 0;
// Resident warps per SM that each FFT pass's launch bounds ask the register
// allocator for (the passes are latency-bound single waves of persistent CTAs).
#ifndef FLP_BATCH_WARPS_R2C
#define FLP_BATCH_WARPS_R2C 24
#endif
#ifndef FLP_BATCH_WARPS_COLS
#define FLP_BATCH_WARPS_COLS 16
#endif
#ifndef FLP_BATCH_WARPS_C2R
#define FLP_BATCH_WARPS_C2R 20
#endif
#ifndef FLP_BATCH_GBY
#define FLP_BATCH_GBY 2
#endif
constexpr int BATCH_GBY = FLP_BATCH_GBY;  // destination rows per thread in the batched gather (64x32 tiles)
constexpr int ROW_SIZES[] = {16, 24, 32, 48, 64, 96, 128, 192, 256};
constexpr int COL_SIZES[] = {32, 48, 64, 96, 128, 192, 256, 384, 512};
constexpr int NSTAGE = 5;
constexpr int BATCH_GRAPH_STEPS = 8;

int row_class(int M) {
    for (int i = 0; i < int(sizeof(ROW_SIZES) / sizeof(int)); ++i)
        if (ROW_SIZES[i] == M) return i;
    return -1;
}
int col_class(int H) {
    for (int i = 0; i < int(sizeof(COL_SIZES) / sizeof(int)); ++i)
        if (COL_SIZES[i] == H) return i;
    return -1;
}
int row_nr(int M, int wpc) {
    switch (M) {
#define X(n) case n: return wpc == 4 ? WRowCfg<n, 4>::NRC : WRowCfg<n, 8>::NRC;
        FLP_ROW_SIZES(X)
#undef X
    }
    return 1;
}
int col_nc(int H) {
    switch (H) {
#define X(n) case n: return WColCfg<n, BATCH_WPC_COLS>::NCC;
        FLP_COL_SIZES(X)
#undef X
    }
    return 1;
}

struct BWorld {
    int W, H, C, K, nsrc, mcls, hcls, pad;
    long long offA;  // float offset of channel 0 in the state / U / DX / DY pools
    long long offS;  // float2 offset in the source-spectrum pool
    long long offT;  // float2 offset in the product pool
    long long offKH; // float2 offset in the kernel-spectrum pool, shared by worlds with the same grid and stencils
    int offKd;       // first kernel descriptor (and spectrum slot) of the world
    int offSrc;      // first source-channel entry
    int twM, twW, twH;
    int pad2;
    FlowParams fp;
};

constexpr int NCLS = 9;  // size classes per FFT pass
// Queue index: FFT stages s in {0,1,2} use queue s*NCLS + class; the flow
// uses one queue per channel count (QF + C for C = 1..4, QF for the rest,
// each with its own compiled kernel); the gather uses QG.
constexpr int NFLOWQ = 5;
constexpr int QF = 3 * NCLS;
constexpr int QG = QF + NFLOWQ;
constexpr int NQUEUE = QG + 1;
inline int flow_queue(int C) { return QF + (C <= 4 ? C : 0); }

struct Pools {
    const BWorld* worlds;
    const int2* items;       // all queues back to back
    const int* q_off;        // NQUEUE+1 offsets into items (device)
    int* counters;           // NQUEUE work-queue counters, zeroed at the start of each step
    int* dmax;      // per-world largest displacement (float bits)
    int* status;
    int n_worlds;
    const float* A;
    float* Anext;
    float* U;
    float* DX;
    float* DY;
    float2* S;
    float2* T;
    const float2* KH;
    const KDesc* kd;
    const int* srcs;
    const int* slots;
    const float2* tw;
};

// A persistent CTA's cursor on a work queue.  Item k's index sits in
// slot[k & 1]; thread 0 claims the following item (atomicAdd on the queue's
// counter) while item k is processed and publishes it at the item's end, so
// the atomic's round trip is hidden behind the item and one barrier per item
// suffices: a slot is rewritten only after every thread has passed the
// barrier that followed its last read.  Each CTA claims up to two indices past
// the end; the counters are rearmed every step.
struct QueueCursor {
    int* counter;
    int n, k, ahead;
    int* slot;  // two shared ints
    __device__ __forceinline__ QueueCursor(int* c, int n_, int* s) : counter(c), n(n_), k(0), ahead(0), slot(s) {
        if (threadIdx.x == 0) {
            slot[0] = atomicAdd(counter, 1);
            ahead = atomicAdd(counter, 1);
        }
        __syncthreads();
    }
    // The current item, -1 when the queue is drained (uniform over the CTA).
    __device__ __forceinline__ int item() const {
        const int it = slot[k & 1];
        return it < n ? it : -1;
    }
    // Publish the claimed item and claim the one after it; call at the end of
    // an item by every thread.
    __device__ __forceinline__ void advance() {
        if (threadIdx.x == 0) {
            slot[(k + 1) & 1] = ahead;
            ahead = atomicAdd(counter, 1);
        }
        ++k;
        __syncthreads();
    }
};


// Wrap-padding of kernel stencils onto W x H planes (Kernel::pad_to_size,
// kernel.rs:98-117), one block per plane: desc[p] = (tap offset, side, plane).
// The planes start zeroed; with a side no larger than the grid every tap lands
// on its own cell, so the scatter equals the reference's sequential writes.
__global__ void k_pad_taps(const float* __restrict__ taps, const int4* __restrict__ desc, float* __restrict__ out,
                           int W, int H) {
    const int4 d = desc[blockIdx.x];
    const int side = d.y, c = side / 2;
    float* o = out + size_t(d.z) * W * H;
    for (int t = threadIdx.x; t < side * side; t += blockDim.x) {
        const int ky = t / side, kx = t - ky * side;
        o[size_t((ky - c + H) % H) * W + (kx - c + W) % W] = taps[d.x + t];
    }
}

// Zero every queue counter and every world's displacement slot.
__global__ void k_batch_reset(Pools p) {
    dep_enter();
    for (int i = threadIdx.x; i < NQUEUE; i += blockDim.x) p.counters[i] = 0;
    for (int i = threadIdx.x; i < p.n_worlds; i += blockDim.x) p.dmax[i] = 0;
}

template <int M>
__global__ void __launch_bounds__(32 * BATCH_WPC_R2C, FLP_BATCH_WARPS_R2C / BATCH_WPC_R2C) k_batch_r2c(Pools p, int q) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    const int base = p.q_off[q], n = p.q_off[q + 1] - base;
    __shared__ int qslot[2];
    for (QueueCursor cur(p.counters + q, n, qslot); cur.item() >= 0; cur.advance()) {
        const int2 item = p.items[base + cur.item()];
        const BWorld w = p.worlds[item.x];
        const int slot = item.y >> 16, g = item.y & 0xFFFF;
        const int c = p.srcs[w.offSrc + slot];
        const size_t N = size_t(2 * M) * w.H;
        float2* Sc = p.S + w.offS + size_t(slot) * (M + 1) * w.H;
        r2c_rows_witem<M, BATCH_WPC_R2C>(fsm, p.A + w.offA + size_t(c) * N, Sc, w.H, g * WRowCfg<M, BATCH_WPC_R2C>::NRC,
                                     p.tw + w.twM, p.tw + w.twW);
    }
}

template <int H>
__global__ void __launch_bounds__(32 * BATCH_WPC_COLS, FLP_BATCH_WARPS_COLS / BATCH_WPC_COLS) k_batch_cols(Pools p, int q) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    const int base = p.q_off[q], n = p.q_off[q + 1] - base;
    __shared__ int qslot[2];
    for (QueueCursor cur(p.counters + q, n, qslot); cur.item() >= 0; cur.advance()) {
        const int2 item = p.items[base + cur.item()];
        const BWorld w = p.worlds[item.x];
        const int u = item.y >> 16, g = item.y & 0xFFFF;  // u: source slot (shared) or kernel
        const int Wc = w.W / 2 + 1;
        const int slot = BATCH_SHARE_COLS ? u : p.slots[w.offKd + u];
        const int kb = BATCH_SHARE_COLS ? 0 : u, ke = BATCH_SHARE_COLS ? w.K : u + 1;
        cols_witem<H, BATCH_WPC_COLS>(fsm, p.S + w.offS + size_t(slot) * Wc * H, p.KH + w.offKH, p.T + w.offT,
                                      p.slots + w.offKd, kb, ke, slot, Wc, g * WColCfg<H, BATCH_WPC_COLS>::NCC,
                                      p.tw + w.twH);
    }
}

template <int M>
__global__ void __launch_bounds__(32 * BATCH_WPC_C2R, FLP_BATCH_WARPS_C2R / BATCH_WPC_C2R) k_batch_c2r(Pools p, int q) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    const int base = p.q_off[q], n = p.q_off[q + 1] - base;
    __shared__ int qslot[2];
    for (QueueCursor cur(p.counters + q, n, qslot); cur.item() >= 0; cur.advance()) {
        const int2 item = p.items[base + cur.item()];
        const BWorld w = p.worlds[item.x];
        const int c = item.y >> 16, g = item.y & 0xFFFF;
        float* Uc = p.U + w.offA + size_t(c) * (2 * M) * w.H;
        c2r_growth_witem<M, BATCH_WPC_C2R>(fsm, p.T + w.offT, p.kd + w.offKd, w.K, c, Uc, w.H,
                                           g * WRowCfg<M, BATCH_WPC_C2R>::NRC, p.tw + w.twM, p.tw + w.twW);
    }
}

// Rows per thread of the batched row-walking flow (tile height 8 * that): the
// persistent kernel is throughput-bound, so a taller walk that reloads fewer
// halo rows pays, where the single-world kernel wants more, shorter tiles.
#ifndef FLP_BATCH_FR_RPT
#define FLP_BATCH_FR_RPT 8
#endif
constexpr int BATCH_FR_RPT = FLP_BATCH_FR_RPT;
constexpr int BATCH_FR_H = 8 * BATCH_FR_RPT;

template <int CV>
__global__ void __launch_bounds__(256) k_batch_flow(Pools p, int q) {
    dep_enter();
    extern __shared__ __align__(16) float sm[];
    const int base = p.q_off[q], n = p.q_off[q + 1] - base;
    __shared__ int qslot[2];
    for (QueueCursor cur(p.counters + q, n, qslot); cur.item() >= 0; cur.advance()) {
        const int2 item = p.items[base + cur.item()];
        const BWorld w = p.worlds[item.x];
        const int tiles_x = (w.W + FL_W - 1) / FL_W;
        const int x0 = (item.y % tiles_x) * FL_W, y0 = (item.y / tiles_x) * (CV ? BATCH_FR_H : FL_H);
        const float* A = p.A + w.offA;
        const float* U = p.U + w.offA;
        float *DX = p.DX + w.offA, *DY = p.DY + w.offA;
        if constexpr (CV == 0)
            flow_item(sm, A, U, DX, DY, w.C, w.W, w.H, w.fp, x0, y0, p.dmax + item.x, p.status);
        else
            flow_rows_item<CV, BATCH_FR_RPT>(A, U, DX, DY, w.W, w.H, w.fp, x0, y0, p.dmax + item.x, p.status);
    }
}

__global__ void __launch_bounds__(256, 3) k_batch_gather(Pools p) {
    dep_enter();
    extern __shared__ __align__(16) float sm[];
    constexpr int q = QG;
    const int base = p.q_off[q], n = p.q_off[q + 1] - base;
    __shared__ int qslot[2];
    for (QueueCursor cur(p.counters + q, n, qslot); cur.item() >= 0; cur.advance()) {
        const int2 item = p.items[base + cur.item()];
        const BWorld w = p.worlds[item.x];
        const int c = item.y >> 16, t = item.y & 0xFFFF;
        const int tiles_x = (w.W + GT_W - 1) / GT_W;
        const int x0 = (t % tiles_x) * GT_W, y0 = (t / tiles_x) * gt_h(BATCH_GBY);
        const size_t off = size_t(w.offA) + size_t(c) * w.W * w.H;
        const int bits = p.dmax[item.x];
        if (w.fp.area_pow2)
            gather_item<true, BATCH_GBY>(sm, p.DX + off, p.DY + off, p.A + off, p.Anext + off, w.W, w.H, w.fp, bits, x0, y0);
        else
            gather_item<false, BATCH_GBY>(sm, p.DX + off, p.DY + off, p.A + off, p.Anext + off, w.W, w.H, w.fp, bits, x0, y0);
    }
}

// FP64 compensated mass per world: one block per world.
__global__ void __launch_bounds__(256) k_batch_mass(const BWorld* worlds, const float* A, double* out) {
    const BWorld w = worlds[blockIdx.x];
    const size_t n = size_t(w.C) * w.W * w.H;
    const float* a = A + w.offA;
    double s = 0.0, c = 0.0;
    for (size_t i = threadIdx.x; i < n; i += 256) {
        const double x = double(a[i]);
        const double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    __shared__ double ss[256], cs[256];
    ss[threadIdx.x] = s;
    cs[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0.0, Cc = 0.0;
        for (int i = 0; i < 256; ++i) {
            const double x = ss[i];
            const double t = S + x;
            if (fabs(S) >= fabs(x)) Cc += (S - t) + x;
            else Cc += (x - t) + S;
            S = t;
            Cc += cs[i];
        }
        out[blockIdx.x] = S + Cc;
    }
}

template <class T>
T* dalloc_b(size_t n) {
    void* p = nullptr;
    throw_cuda(flp::dmalloc(&p, (n ? n : 1) * sizeof(T)), "cudaMalloc");
    return static_cast<T*>(p);
}

void ckb(cudaError_t e, const char* what) { throw_cuda(e, what); }

std::once_flag g_battr_once;

// Per-class launch helpers (class index -> template instantiation).
const void* r2c_fn(int cls) {
    switch (ROW_SIZES[cls]) {
#define X(n) case n: return (const void*)k_batch_r2c<n>;
        FLP_ROW_SIZES(X)
#undef X
    }
    return nullptr;
}
const void* c2r_fn(int cls) {
    switch (ROW_SIZES[cls]) {
#define X(n) case n: return (const void*)k_batch_c2r<n>;
        FLP_ROW_SIZES(X)
#undef X
    }
    return nullptr;
}
const void* cols_fn(int cls) {
    switch (COL_SIZES[cls]) {
#define X(n) case n: return (const void*)k_batch_cols<n>;
        FLP_COL_SIZES(X)
#undef X
    }
    return nullptr;
}
size_t r2c_smem(int cls) {
    switch (ROW_SIZES[cls]) {
#define X(n) case n: return WRowCfg<n, BATCH_WPC_R2C>::smem_r2c;
        FLP_ROW_SIZES(X)
#undef X
    }
    return 0;
}
size_t c2r_smem(int cls) {
    switch (ROW_SIZES[cls]) {
#define X(n) case n: return WRowCfg<n, BATCH_WPC_C2R>::smem_c2r;
        FLP_ROW_SIZES(X)
#undef X
    }
    return 0;
}
size_t cols_smem(int cls) {
    switch (COL_SIZES[cls]) {
#define X(n) case n: return WColCfg<n, BATCH_WPC_COLS>::smem;
        FLP_COL_SIZES(X)
#undef X
    }
    return 0;
}

}  // namespace
}  // namespace flp

using namespace flp;

// ---- per-world statistics of the channel sum (fitness evaluation) ----------
// S = sum_c A_c per cell, channels added in order as SimulationState::
// channel_sum does (propagator.rs:109-120); every reduction is FP64.
__device__ __forceinline__ float chan_sum(const float* a, size_t N, int C, size_t i) {
    float s = 0.f;
    for (int c = 0; c < C; ++c) s = __fadd_rn(s, a[size_t(c) * N + i]);
    return s;
}

template <int NV>
__device__ __forceinline__ void block_sum_nd(double (&v)[NV], double (*red)[NV]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[warp][k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w][k];
        v[k] = t;
    }
}

// One CTA per world.  Writes FLP_BATCH_NSTAT doubles: total of S, total of
// S > 0, centre of mass (x, y) of S > 0 (the grid centre when that total is at
// most 1e-6), radius (second moment about it), max(0, max S), #(S > 1e-6),
// #(S < 0), mean, variance, mean neighbour difference (left and up, no wrap,
// over 2N), N (fitness.rs:195-240, 420-520).
__global__ void __launch_bounds__(256) k_batch_stats(const BWorld* worlds, const float* A, double* out) {
    __shared__ double red[8][8];
    __shared__ float redm[8];
    const BWorld w = worlds[blockIdx.x];
    const size_t N = size_t(w.W) * w.H;
    const float* a = A + w.offA;
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // total, pos, xm, ym, active, neg, grad, -
    float mx = 0.f;
    for (size_t i = threadIdx.x; i < N; i += blockDim.x) {
        const int x = int(i % w.W), y = int(i / w.W);
        const float S = chan_sum(a, N, w.C, i);
        v[0] += S;
        if (S > 0.f) {
            v[1] += S;
            v[2] += double(x) * S;
            v[3] += double(y) * S;
        }
        mx = fmaxf(mx, S);
        v[4] += S > 1e-6f ? 1.0 : 0.0;
        v[5] += S < 0.f ? 1.0 : 0.0;
        if (x > 0) v[6] += fabs(double(S) - double(chan_sum(a, N, w.C, i - 1)));
        if (y > 0) v[6] += fabs(double(S) - double(chan_sum(a, N, w.C, i - w.W)));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) redm[threadIdx.x >> 5] = mx;
    block_sum_nd<8>(v, red);
    for (int k = 0; k < int(blockDim.x >> 5); ++k) mx = fmaxf(mx, redm[k]);
    const bool has = v[1] > 1e-6;
    const double cx = has ? v[2] / v[1] : 0.5 * w.W, cy = has ? v[3] / v[1] : 0.5 * w.H;
    const double mean = v[0] / double(N);
    double u[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // moment, sum of squared deviations
    for (size_t i = threadIdx.x; i < N; i += blockDim.x) {
        const double x = double(i % w.W), y = double(i / w.W);
        const double S = chan_sum(a, N, w.C, i);
        if (S > 0.0) u[0] += S * ((x - cx) * (x - cx) + (y - cy) * (y - cy));
        u[1] += (S - mean) * (S - mean);
    }
    block_sum_nd<8>(u, red);
    if (threadIdx.x == 0) {
        double* o = out + size_t(blockIdx.x) * FLP_BATCH_NSTAT;
        o[0] = v[0];
        o[1] = v[1];
        o[2] = cx;
        o[3] = cy;
        o[4] = has ? sqrt(u[0] / v[1]) : 0.0;
        o[5] = double(mx);
        o[6] = v[4];
        o[7] = v[5];
        o[8] = mean;
        o[9] = u[1] / double(N);
        o[10] = v[6] / (2.0 * double(N));
        o[11] = double(N);
    }
}

// Channel sums of every world into snapshot slot `slot` (cells of world w at
// cell_off[w]).
__global__ void __launch_bounds__(256) k_batch_snapshot(const BWorld* worlds, const float* A,
                                                        const long long* cell_off, float* snaps, size_t cells,
                                                        int slot) {
    const BWorld w = worlds[blockIdx.x];
    const size_t N = size_t(w.W) * w.H;
    float* dst = snaps + size_t(slot) * cells + size_t(cell_off[blockIdx.x]);
    for (size_t i = threadIdx.x; i < N; i += blockDim.x) dst[i] = chan_sum(A + w.offA, N, w.C, i);
}

// Normalised dot product of two snapshots of every world (fitness.rs:337-350),
// 0 when either norm is at most 1e-6.
__global__ void __launch_bounds__(256) k_batch_similarity(const BWorld* worlds, const long long* cell_off,
                                                          const float* snaps, size_t cells, int sa, int sb,
                                                          double* out) {
    __shared__ double red[8][4];
    const BWorld w = worlds[blockIdx.x];
    const size_t N = size_t(w.W) * w.H;
    const float* pa = snaps + size_t(sa) * cells + size_t(cell_off[blockIdx.x]);
    const float* pb = snaps + size_t(sb) * cells + size_t(cell_off[blockIdx.x]);
    double v[4] = {0, 0, 0, 0};
    for (size_t i = threadIdx.x; i < N; i += blockDim.x) {
        const double x = pa[i], y = pb[i];
        v[0] += x * y;
        v[1] += x * x;
        v[2] += y * y;
    }
    block_sum_nd<4>(v, red);
    if (threadIdx.x == 0) {
        const double na = sqrt(v[1]), nb = sqrt(v[2]);
        out[blockIdx.x] = (na > 1e-6 && nb > 1e-6) ? v[0] / (na * nb) : 0.0;
    }
}

struct flp_batch {
    std::vector<SimulationConfig> cfgs;
    std::vector<BWorld> hw;
    int n = 0;
    size_t cells_total = 0;  // sum of C*N
    int unique_spectra = 0;  // distinct kernel-spectrum sets in the pool
    size_t kh_bytes = 0;
    size_t kh_cap = 0;       // float2 allocated for KH
    cudaStream_t st = nullptr;
    BWorld* d_worlds = nullptr;
    int2* d_items = nullptr;
    int* d_qoff = nullptr;
    int n_q[NQUEUE] = {0};
    int* d_counters = nullptr;
    int* d_dmax = nullptr;
    int* d_status = nullptr;
    float* A[2] = {nullptr, nullptr};
    float *U = nullptr, *DX = nullptr, *DY = nullptr;
    float2 *S = nullptr, *T = nullptr, *KH = nullptr, *tw = nullptr;
    KDesc* d_kd = nullptr;
    int *d_srcs = nullptr, *d_slots = nullptr;
    double* d_mass = nullptr;
    double* d_stats = nullptr;        // n x FLP_BATCH_NSTAT
    long long* d_celloff = nullptr;   // first cell of each world in a snapshot slot
    float* d_snaps = nullptr;         // n_snap slots of sum_w W*H floats
    int n_snap = 0;
    size_t cells = 0;                 // sum over worlds of W*H
    int cur = 0;
    const void* q_fn[NQUEUE] = {nullptr};
    int q_grid[NQUEUE] = {0};
    int q_block[NQUEUE] = {0};
    size_t q_smem[NQUEUE] = {0};
    std::vector<float> time;
    std::vector<uint64_t> steps;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaEvent_t ev[NSTAGE + 1] = {nullptr};
    std::vector<cudaEvent_t> pev;  // per-step event ring of the profiling entry
    // The size-class kernels of one stage are independent: all but the first
    // run on side streams forked from and joined back into st, so that in the
    // captured graph they are parallel branches that fill each other's tails.
    static constexpr int NSIDE = NCLS - 1;
    cudaStream_t side[NSIDE] = {nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[NSIDE] = {nullptr};
    void* flush_buf = nullptr;
    size_t flush_bytes = 0;

    Pools pools() const {
        Pools p{};
        p.worlds = d_worlds;
        p.items = d_items;
        p.q_off = d_qoff;
        p.counters = d_counters;
        p.dmax = d_dmax;
        p.status = d_status;
        p.n_worlds = n;
        p.A = A[cur];
        p.Anext = A[cur ^ 1];
        p.U = U; p.DX = DX; p.DY = DY;
        p.S = S; p.T = T; p.KH = KH;
        p.kd = d_kd; p.srcs = d_srcs; p.slots = d_slots; p.tw = tw;
        return p;
    }

    // Queue kernels are launched with programmatic stream serialization (they
    // begin with dep_enter), so each one's blocks are placed while its
    // predecessor drains.
    void launch_queue(int q, Pools& p, cudaStream_t qs) {
        if (!n_q[q]) return;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(q_grid[q]);
        cfg.blockDim = dim3(q_block[q]);
        cfg.dynamicSmemBytes = q_smem[q];
        cfg.stream = qs;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int qq = q;
        void* args2[] = {&p, &qq};
        void* args1[] = {&p};
        ckb(cudaLaunchKernelExC(&cfg, q_fn[q], q < QG ? args2 : args1), "batch launch");
    }

    // reset, then per stage the size-class kernels of that stage
    // evs (NSTAGE + 1 events, optional): evs[0] before the step, evs[NSTAGE]
    // after it and, when staged, evs[1..NSTAGE-1] between the stages.
    // The non-empty queues q0 .. q0+nq-1 of one stage: the first on st, the
    // others forked onto side streams and joined back.
    void launch_stage(int q0, int nq, Pools& p) {
        int act[NCLS], na = 0;
        for (int q = q0; q < q0 + nq; ++q)
            if (n_q[q]) act[na++] = q;
        if (na > 1) ckb(cudaEventRecord(ev_fork, st), "event");
        for (int k = 1; k < na; ++k) {
            ckb(cudaStreamWaitEvent(side[k - 1], ev_fork, 0), "fork");
            launch_queue(act[k], p, side[k - 1]);
            ckb(cudaEventRecord(ev_join[k - 1], side[k - 1]), "event");
        }
        if (na > 0) launch_queue(act[0], p, st);
        for (int k = 1; k < na; ++k) ckb(cudaStreamWaitEvent(st, ev_join[k - 1], 0), "join");
    }

    void enqueue_step(cudaEvent_t* evs = nullptr, bool staged = false) {
        Pools p = pools();
        if (evs) ckb(cudaEventRecord(evs[0], st), "event");
        launch_dep(k_batch_reset, 1, 256, 0, st, p);
        for (int stage = 0; stage < 3; ++stage) {
            launch_stage(stage * NCLS, NCLS, p);
            if (evs && staged) ckb(cudaEventRecord(evs[stage + 1], st), "event");
        }
        launch_stage(QF, NFLOWQ, p);
        if (evs && staged) ckb(cudaEventRecord(evs[4], st), "event");
        launch_queue(QG, p, st);
        if (evs) ckb(cudaEventRecord(evs[5], st), "event");
        ckb(cudaGetLastError(), "batch launch");
        cur ^= 1;
    }

    void advance(uint64_t k) {
        for (int w = 0; w < n; ++w) {
            for (uint64_t i = 0; i < k; ++i) time[w] += cfgs[w].dt;
            steps[w] += k;
        }
    }

    void drop_graphs() {
        for (auto& g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    void free_all() {
        drop_graphs();
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : pev) cudaEventDestroy(e);
        pev.clear();
        for (cudaEvent_t e : ev_join)
            if (e) cudaEventDestroy(e);
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (cudaStream_t q : side)
            if (q) cudaStreamDestroy(q);
        void* ptrs[] = {d_worlds, d_items, d_qoff, d_counters, d_dmax, d_status, A[0], A[1], U, DX, DY, S, T,
                        KH, tw, d_kd, d_srcs, d_slots, d_mass, flush_buf, d_stats, d_celloff, d_snaps};
        for (void* q : ptrs)
            if (q) flp::dfree(q);
        if (st) cudaStreamDestroy(st);
    }
};

namespace flp {
namespace {

// The kernel descriptor of one kernel (growth parameters and stencil radius).
KDesc make_kdesc(const KernelConfig& kc, int radius) {
    KDesc k{};
    k.src = kc.source_channel;
    k.tgt = kc.target_channel;
    k.r = radius;
    k.weight = kc.weight;
    k.mu = kc.mu;
    const float sigma_sq_2 = 2.0f * kc.sigma * kc.sigma;
    k.inv2s2 = 1.0f / sigma_sq_2;
    return k;
}

// Kernel spectra depend only on the grid and the stencils: the key of a
// world's spectrum set.
std::string kh_key(int W, int H, const std::vector<KernelStencil>& st) {
    std::string key = std::to_string(W) + "x" + std::to_string(H);
    for (const KernelStencil& ks : st) {
        key += "|" + std::to_string(ks.size) + ":";
        key.append(reinterpret_cast<const char*>(ks.data.data()), ks.data.size() * sizeof(float));
    }
    return key;
}

// The stencils of world w's config, each checked against the grid like
// pad_kernel (kernel.rs:98-117).
std::vector<KernelStencil> world_stencils(const SimulationConfig& c, int w) {
    std::vector<KernelStencil> out;
    for (const KernelConfig& kc : c.kernels) {
        out.push_back(build_kernel(kc, c.kernel_radius, 2));
        if (out.back().radius > c.width || out.back().radius > c.height)
            throw ConfigError("world " + std::to_string(w) + ": kernel radius " + std::to_string(out.back().radius) +
                              " exceeds a grid side");
    }
    return out;
}

void batch_spectra(flp_batch* b, const std::vector<std::vector<KernelStencil>>& stencils,
                   const std::vector<char>& kh_owner);

void batch_create(flp_batch* b, const char* const* jsons, int n) {
    if (n <= 0) throw std::invalid_argument("need at least one world");
    std::call_once(g_battr_once, [] {
        auto set = [](const void* f, size_t bytes) {
            cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
            cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        };
        for (int c = 0; c < NCLS; ++c) {
            set(r2c_fn(c), r2c_smem(c));
            set(c2r_fn(c), c2r_smem(c));
            set(cols_fn(c), cols_smem(c));
        }
        set((const void*)k_batch_flow<0>, flow_smem_bytes_inl(64));
        set((const void*)k_batch_gather, gather_smem_bytes_inl(BATCH_GBY));
        transport_2d_set_attributes();
        fft2d_set_attributes(200 * 1024);
    });
    b->n = n;
    ckb(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking), "stream");
    for (auto& e : b->ev) ckb(cudaEventCreate(&e), "event");
    for (auto& q : b->side) ckb(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking), "stream");
    ckb(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming), "event");
    for (auto& e : b->ev_join) ckb(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    // ---- per-world layout
    std::vector<KDesc> kd;
    std::vector<int> srcs, slots;
    std::vector<float2> tw;
    std::vector<std::pair<int, int>> tw_index;  // (L, offset) tables exp(-2 pi i t / L), t < L
    auto twiddles = [&](int L) {
        for (auto& e : tw_index)
            if (e.first == L) return e.second;
        const int off = int(tw.size());
        for (int t = 0; t < L; ++t) {
            const double ang = -2.0 * M_PI * double(t) / double(L);
            tw.push_back(make_float2(float(std::cos(ang)), float(std::sin(ang))));
        }
        tw_index.push_back({L, off});
        return off;
    };
    long long offA = 0, offS = 0, offT = 0, offKH = 0;
    // Kernel spectra depend only on the grid and the stencils: worlds that
    // share both (a parameter sweep over growth, flow or dt) share one set.
    std::map<std::string, long long> kh_of;
    std::vector<char> kh_owner(n, 0);
    int cmax = 1;
    // parsing, the per-world checks and the kernel stencils are independent
    // per world: host threads
    std::vector<SimulationConfig> parsed(n);
    std::vector<std::vector<KernelStencil>> stencils(n);
    parallel_for(n, [&](int w) {
        if (!jsons[w]) throw ConfigError("null config for world " + std::to_string(w));
        SimulationConfig c = parse_config(jsons[w]);
        if (c.is_3d()) throw ConfigError("world " + std::to_string(w) + ": the batched engine serves 2D worlds");
        const int mcls = (c.width % 2 == 0) ? row_class(c.width / 2) : -1;
        if (mcls < 0 || col_class(c.height) < 0)
            throw ConfigError("world " + std::to_string(w) + ": batched sides must be even widths with W/2 in {16..256} and H in {32..512} of factors 2 and 3");
        stencils[w] = world_stencils(c, w);
        parsed[w] = std::move(c);
    });
    for (int w = 0; w < n; ++w) {
        const SimulationConfig& c = parsed[w];
        BWorld d{};
        d.W = c.width; d.H = c.height; d.C = c.channels; d.K = int(c.kernels.size());
        d.mcls = row_class(d.W / 2);
        d.hcls = col_class(d.H);
        cmax = std::max(cmax, d.C);
        d.offA = offA;
        offA += (long long)d.C * d.W * d.H;
        d.offKd = int(kd.size());
        d.offSrc = int(srcs.size());
        std::vector<int> my_src;
        for (int k = 0; k < d.K; ++k) {
            const KernelConfig& kc = c.kernels[k];
            kd.push_back(make_kdesc(kc, stencils[w][k].radius));
            auto it = std::find(my_src.begin(), my_src.end(), kc.source_channel);
            int slot;
            if (it == my_src.end()) { slot = int(my_src.size()); my_src.push_back(kc.source_channel); }
            else slot = int(it - my_src.begin());
            slots.push_back(slot);
        }
        d.nsrc = int(my_src.size());
        srcs.insert(srcs.end(), my_src.begin(), my_src.end());
        const long long spec = (long long)(d.W / 2 + 1) * d.H;
        d.offS = offS;
        offS += spec * std::max(d.nsrc, 1);
        d.offT = offT;
        offT += spec * std::max(d.K, 1);
        {
            std::string key = kh_key(d.W, d.H, stencils[w]);
            auto it = kh_of.find(key);
            if (it != kh_of.end()) {
                d.offKH = it->second;
            } else {
                d.offKH = offKH;
                kh_of.emplace(key, offKH);
                kh_owner[w] = 1;
                offKH += spec * std::max(d.K, 1);
            }
        }
        d.twM = twiddles(d.W / 2);
        d.twW = twiddles(d.W);
        d.twH = twiddles(d.H);
        d.fp = flow_params_of(c);
        b->hw.push_back(d);
        b->cfgs.push_back(c);
    }
    b->cells_total = size_t(offA);
    b->time.assign(n, 0.f);
    b->steps.assign(n, 0);
    // ---- pools
    const size_t CN = size_t(offA);
    b->A[0] = dalloc_b<float>(CN);
    b->A[1] = dalloc_b<float>(CN);
    b->U = dalloc_b<float>(CN);
    b->DX = dalloc_b<float>(CN);
    b->DY = dalloc_b<float>(CN);
    ckb(cudaMemsetAsync(b->A[0], 0, CN * sizeof(float), b->st), "memset");
    ckb(cudaMemsetAsync(b->A[1], 0, CN * sizeof(float), b->st), "memset");
    ckb(cudaMemsetAsync(b->U, 0, CN * sizeof(float), b->st), "memset");
    b->S = dalloc_b<float2>(size_t(offS));
    b->T = dalloc_b<float2>(size_t(offT));
    b->KH = dalloc_b<float2>(size_t(offKH));
    b->unique_spectra = int(kh_of.size());
    b->kh_bytes = size_t(offKH) * sizeof(float2);
    b->kh_cap = size_t(offKH);
    b->tw = dalloc_b<float2>(tw.size());
    b->d_kd = dalloc_b<KDesc>(kd.size());
    b->d_srcs = dalloc_b<int>(srcs.size());
    b->d_slots = dalloc_b<int>(slots.size());
    b->d_worlds = dalloc_b<BWorld>(n);
    b->d_counters = dalloc_b<int>(NQUEUE);
    b->d_dmax = dalloc_b<int>(n);
    b->d_status = dalloc_b<int>(1);
    b->d_mass = dalloc_b<double>(n);
    b->d_stats = dalloc_b<double>(size_t(n) * FLP_BATCH_NSTAT);
    {
        std::vector<long long> co(n);
        long long acc = 0;
        for (int w = 0; w < n; ++w) {
            co[w] = acc;
            acc += (long long)b->hw[w].W * b->hw[w].H;
        }
        b->cells = size_t(acc);
        b->d_celloff = dalloc_b<long long>(n);
        ckb(cudaMemcpy(b->d_celloff, co.data(), n * sizeof(long long), cudaMemcpyHostToDevice), "copy");
    }
    ckb(cudaMemsetAsync(b->d_counters, 0, NQUEUE * sizeof(int), b->st), "memset");
    ckb(cudaMemsetAsync(b->d_status, 0, sizeof(int), b->st), "memset");
    ckb(cudaMemcpy(b->tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice), "copy");
    if (!kd.empty()) ckb(cudaMemcpy(b->d_kd, kd.data(), kd.size() * sizeof(KDesc), cudaMemcpyHostToDevice), "copy");
    if (!srcs.empty()) ckb(cudaMemcpy(b->d_srcs, srcs.data(), srcs.size() * sizeof(int), cudaMemcpyHostToDevice), "copy");
    if (!slots.empty()) ckb(cudaMemcpy(b->d_slots, slots.data(), slots.size() * sizeof(int), cudaMemcpyHostToDevice), "copy");
    ckb(cudaMemcpy(b->d_worlds, b->hw.data(), n * sizeof(BWorld), cudaMemcpyHostToDevice), "copy");
    batch_spectra(b, stencils, kh_owner);
    // ---- work queues, largest worlds first
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return size_t(b->hw[a].W) * b->hw[a].H > size_t(b->hw[c].W) * b->hw[c].H;
    });
    std::vector<int2> items[NQUEUE];
    for (int w : order) {
        const BWorld& d = b->hw[w];
        const int nr = row_nr(d.W / 2, BATCH_WPC_R2C), nr2 = row_nr(d.W / 2, BATCH_WPC_C2R), nc = col_nc(d.H),
                  Wc = d.W / 2 + 1;
        for (int s2 = 0; s2 < d.nsrc; ++s2)
            for (int g = 0; g < (d.H + nr - 1) / nr; ++g) items[0 * NCLS + d.mcls].push_back(make_int2(w, (s2 << 16) | g));
        for (int u = 0; u < (BATCH_SHARE_COLS ? d.nsrc : d.K); ++u)
            for (int g = 0; g < (Wc + nc - 1) / nc; ++g) items[1 * NCLS + d.hcls].push_back(make_int2(w, (u << 16) | g));
        for (int c = 0; c < d.C; ++c)
            for (int g = 0; g < (d.H + nr2 - 1) / nr2; ++g) items[2 * NCLS + d.mcls].push_back(make_int2(w, (c << 16) | g));
        const int fth = d.C <= 4 ? BATCH_FR_H : FL_H;
        const int ftiles = ((d.W + FL_W - 1) / FL_W) * ((d.H + fth - 1) / fth);
        for (int t = 0; t < ftiles; ++t) items[flow_queue(d.C)].push_back(make_int2(w, t));
        const int gtiles = ((d.W + GT_W - 1) / GT_W) * ((d.H + gt_h(BATCH_GBY) - 1) / gt_h(BATCH_GBY));
        for (int c = 0; c < d.C; ++c)
            for (int t = 0; t < gtiles; ++t) items[QG].push_back(make_int2(w, (c << 16) | t));
    }
    std::vector<int2> all;
    std::vector<int> qoff(NQUEUE + 1, 0);
    for (int q = 0; q < NQUEUE; ++q) {
        qoff[q] = int(all.size());
        all.insert(all.end(), items[q].begin(), items[q].end());
        b->n_q[q] = int(items[q].size());
    }
    qoff[NQUEUE] = int(all.size());
    b->d_items = dalloc_b<int2>(all.size());
    b->d_qoff = dalloc_b<int>(qoff.size());
    if (!all.empty()) ckb(cudaMemcpy(b->d_items, all.data(), all.size() * sizeof(int2), cudaMemcpyHostToDevice), "copy");
    ckb(cudaMemcpy(b->d_qoff, qoff.data(), qoff.size() * sizeof(int), cudaMemcpyHostToDevice), "copy");
    // ---- persistent grids: one wave of resident CTAs per queue
    int dev = 0, sms = 0;
    ckb(cudaGetDevice(&dev), "device");
    ckb(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attr");
    for (int q = 0; q < NQUEUE; ++q) {
        const int stage = q < QF ? q / NCLS : (q < QG ? 3 : 4);
        const int cls = q % NCLS;
        switch (stage) {
            case 0: b->q_fn[q] = r2c_fn(cls); b->q_smem[q] = r2c_smem(cls); break;
            case 1: b->q_fn[q] = cols_fn(cls); b->q_smem[q] = cols_smem(cls); break;
            case 2: b->q_fn[q] = c2r_fn(cls); b->q_smem[q] = c2r_smem(cls); break;
            case 3: {
                const void* fns[NFLOWQ] = {(const void*)k_batch_flow<0>, (const void*)k_batch_flow<1>,
                                           (const void*)k_batch_flow<2>, (const void*)k_batch_flow<3>,
                                           (const void*)k_batch_flow<4>};
                b->q_fn[q] = fns[q - QF];
                b->q_smem[q] = q == QF ? flow_smem_bytes_inl(cmax) : 0;
                break;
            }
            default: b->q_fn[q] = (const void*)k_batch_gather; b->q_smem[q] = gather_smem_bytes_inl(BATCH_GBY); break;
        }
        if (!b->n_q[q]) continue;
        int per_sm = 0;
        const int pass = q < 3 * NCLS ? q / NCLS : 3;
        b->q_block[q] = pass == 0 ? 32 * BATCH_WPC_R2C : pass == 1 ? 32 * BATCH_WPC_COLS
                      : pass == 2 ? 32 * BATCH_WPC_C2R : 256;
        ckb(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->q_fn[q], b->q_block[q], b->q_smem[q]),
            "occupancy");
        b->q_grid[q] = std::max(1, std::min(per_sm * sms, b->n_q[q]));
    }
    ckb(cudaStreamSynchronize(b->st), "sync");
}

// Kernel spectra with the single-world FFT passes, one launch pair per grid
// size (in chunks): the stencils are wrap-padded on the device and each
// world's spectra are copied to its place in the pool (worlds with kh_owner
// set own a set; the others share one); one synchronisation at the end.
void batch_spectra(flp_batch* b, const std::vector<std::vector<KernelStencil>>& stencils,
                   const std::vector<char>& kh_owner) {
    const int n = b->n;
    {
        std::map<std::pair<int, int>, std::vector<int>> groups;
        for (int w = 0; w < n; ++w)
            if (b->hw[w].K > 0 && kh_owner[w]) groups[{b->hw[w].W, b->hw[w].H}].push_back(w);
        DevScratch scratch;
        // one scratch region for every size and chunk, reused in stream order:
        // padded planes, their row spectra and their full spectra
        size_t cap_pad = 0, cap_spec = 0;
        for (const auto& gr : groups) {
            const size_t plane = size_t(gr.first.first) * gr.first.second;
            const size_t spec = size_t(gr.first.first / 2 + 1) * gr.first.second;
            const size_t max_planes = std::max<size_t>(1, (size_t(64) << 20) / plane);
            size_t group_planes = 0, kmax = 0;
            for (int w : gr.second) {
                group_planes += size_t(b->hw[w].K);
                kmax = std::max(kmax, size_t(b->hw[w].K));
            }
            const size_t cap = std::max(kmax, std::min(group_planes, max_planes));
            cap_pad = std::max(cap_pad, cap * plane);
            cap_spec = std::max(cap_spec, cap * spec);
        }
        float* d_pad = groups.empty() ? nullptr : scratch.add(dalloc_b<float>(cap_pad));
        float2* d_tmp = groups.empty() ? nullptr : scratch.add(dalloc_b<float2>(cap_spec));
        float2* d_out = groups.empty() ? nullptr : scratch.add(dalloc_b<float2>(cap_spec));
        for (const auto& gr : groups) {
            const int W = gr.first.first, H = gr.first.second;
            const size_t plane = size_t(W) * H, spec = size_t(W / 2 + 1) * H;
            const BWorld& d0 = b->hw[gr.second.front()];
            FftGeom g;
            make_plan(W / 2, g.pm);
            make_plan(H, g.ph);
            g.twM = b->tw + d0.twM;
            g.twW = b->tw + d0.twW;
            g.twH = b->tw + d0.twH;
            const size_t max_planes = std::max<size_t>(1, (size_t(64) << 20) / plane);  // 256 MB of padded planes
            size_t i0 = 0;
            while (i0 < gr.second.size()) {
                // a chunk of worlds of this size
                size_t i1 = i0, planes = 0;
                while (i1 < gr.second.size() && (i1 == i0 || planes + size_t(b->hw[gr.second[i1]].K) <= max_planes))
                    planes += size_t(b->hw[gr.second[i1++]].K);
                std::vector<float> taps;
                std::vector<int4> desc;  // per plane: tap offset, stencil side, plane index, unused
                bool host_pad = false;
                for (size_t i = i0; i < i1; ++i)
                    for (const KernelStencil& ks : stencils[gr.second[i]]) {
                        if (ks.size > W || ks.size > H) host_pad = true;  // wrapped taps overwrite: pad on the host
                        desc.push_back(make_int4(int(taps.size()), ks.size, int(desc.size()), 0));
                        taps.insert(taps.end(), ks.data.begin(), ks.data.end());
                    }
                if (host_pad) {
                    std::vector<float> padded(planes * plane);
                    size_t pi = 0;
                    for (size_t i = i0; i < i1; ++i)
                        for (const KernelStencil& ks : stencils[gr.second[i]]) {
                            const std::vector<float> pk = pad_kernel(ks, W, H, 1);
                            std::copy(pk.begin(), pk.end(), padded.begin() + (pi++) * plane);
                        }
                    ckb(cudaMemcpyAsync(d_pad, padded.data(), padded.size() * sizeof(float), cudaMemcpyHostToDevice,
                                        b->st), "copy");
                    ckb(cudaStreamSynchronize(b->st), "sync");  // the host buffer goes out of scope
                } else {
                    float* d_taps = scratch.add(dalloc_b<float>(taps.size()));
                    int4* d_desc = scratch.add(dalloc_b<int4>(desc.size()));
                    ckb(cudaMemcpyAsync(d_taps, taps.data(), taps.size() * sizeof(float), cudaMemcpyHostToDevice, b->st),
                        "copy");
                    ckb(cudaMemcpyAsync(d_desc, desc.data(), desc.size() * sizeof(int4), cudaMemcpyHostToDevice, b->st),
                        "copy");
                    ckb(cudaMemsetAsync(d_pad, 0, planes * plane * sizeof(float), b->st), "memset");
                    k_pad_taps<<<dim3(unsigned(planes)), 256, 0, b->st>>>(d_taps, d_desc, d_pad, W, H);
                }
                launch_fft_r2c(d_pad, d_tmp, nullptr, int(planes), W, H, g, nullptr, 0, b->st);
                launch_fft_cols(d_tmp, nullptr, d_out, nullptr, int(planes), W, H, g, 1,
                                float(1.0 / (double(W) * double(H))), b->st);
                size_t pi = 0;
                for (size_t i = i0; i < i1; ++i) {
                    const BWorld& d = b->hw[gr.second[i]];
                    ckb(cudaMemcpyAsync(b->KH + d.offKH, d_out + pi * spec, size_t(d.K) * spec * sizeof(float2),
                                        cudaMemcpyDeviceToDevice, b->st), "copy");
                    pi += size_t(d.K);
                }
                ckb(cudaGetLastError(), "kernel spectra");
                i0 = i1;
            }
        }
        ckb(cudaStreamSynchronize(b->st), "sync");
    }
}

// New configs for the worlds of an existing batch (an evolution engine's next
// generation).  Every world keeps its sides, channel count and kernels'
// (source, target) channel pairs, so the pools, the work queues and the
// captured step graphs stay valid; the kernel descriptors, stencils, flow
// parameters and kernel spectra are rebuilt, the states zeroed and the clocks
// reset.  All configs are parsed and checked before anything changes.
void batch_reconfigure(flp_batch* b, const char* const* jsons, int n) {
    if (n != b->n)
        throw std::invalid_argument("reconfigure needs one config per world (" + std::to_string(b->n) + ")");
    ckb(cudaStreamSynchronize(b->st), "sync");
    std::vector<SimulationConfig> cfgs;
    cfgs.reserve(n);
    std::vector<BWorld> hw = b->hw;
    std::vector<KDesc> kd;
    std::vector<std::vector<KernelStencil>> stencils(n);
    std::map<std::string, long long> kh_of;
    std::vector<char> kh_owner(n, 0);
    long long offKH = 0;
    std::vector<SimulationConfig> parsed(n);
    parallel_for(n, [&](int w) {
        if (!jsons[w]) throw ConfigError("null config for world " + std::to_string(w));
        SimulationConfig c = parse_config(jsons[w]);
        const BWorld& d = hw[w];
        const SimulationConfig& old = b->cfgs[w];
        bool same = !c.is_3d() && c.width == d.W && c.height == d.H && c.channels == d.C &&
                    int(c.kernels.size()) == d.K;
        for (int k = 0; same && k < d.K; ++k)
            same = c.kernels[k].source_channel == old.kernels[k].source_channel &&
                   c.kernels[k].target_channel == old.kernels[k].target_channel;
        if (!same)
            throw std::invalid_argument("world " + std::to_string(w) +
                                        ": a reconfigured world keeps its sides, channels and kernel channel pairs");
        stencils[w] = world_stencils(c, w);
        parsed[w] = std::move(c);
    });
    for (int w = 0; w < n; ++w) {
        SimulationConfig& c = parsed[w];
        BWorld& d = hw[w];
        for (int k = 0; k < d.K; ++k) kd.push_back(make_kdesc(c.kernels[k], stencils[w][k].radius));
        const std::string key = kh_key(d.W, d.H, stencils[w]);
        auto it = kh_of.find(key);
        if (it != kh_of.end()) {
            d.offKH = it->second;
        } else {
            d.offKH = offKH;
            kh_of.emplace(key, offKH);
            kh_owner[w] = 1;
            offKH += (long long)(d.W / 2 + 1) * d.H * std::max(d.K, 1);
        }
        d.fp = flow_params_of(c);
        cfgs.push_back(std::move(c));
    }
    if (size_t(offKH) > b->kh_cap) {
        // a larger spectrum pool (allocated first, so that a failure leaves
        // the batch as it was); the captured graphs hold the old pointer
        float2* kh = dalloc_b<float2>(size_t(offKH));
        b->drop_graphs();
        flp::dfree(b->KH);
        b->KH = kh;
        b->kh_cap = size_t(offKH);
    }
    b->hw = std::move(hw);
    b->cfgs = std::move(cfgs);
    b->unique_spectra = int(kh_of.size());
    b->kh_bytes = size_t(offKH) * sizeof(float2);
    if (!kd.empty()) ckb(cudaMemcpy(b->d_kd, kd.data(), kd.size() * sizeof(KDesc), cudaMemcpyHostToDevice), "copy");
    ckb(cudaMemcpy(b->d_worlds, b->hw.data(), n * sizeof(BWorld), cudaMemcpyHostToDevice), "copy");
    const size_t CN = b->cells_total;
    ckb(cudaMemsetAsync(b->A[0], 0, CN * sizeof(float), b->st), "memset");
    ckb(cudaMemsetAsync(b->A[1], 0, CN * sizeof(float), b->st), "memset");
    ckb(cudaMemsetAsync(b->U, 0, CN * sizeof(float), b->st), "memset");
    ckb(cudaMemsetAsync(b->d_status, 0, sizeof(int), b->st), "memset");
    batch_spectra(b, stencils, kh_owner);
    b->time.assign(n, 0.f);
    b->steps.assign(n, 0);
}

void batch_build_graph(flp_batch* b) {
    const int c0 = b->cur;
    cudaGraph_t g = nullptr;
    ckb(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal), "capture");
    try {
        for (int i = 0; i < BATCH_GRAPH_STEPS; ++i) b->enqueue_step();
    } catch (...) {
        cudaStreamEndCapture(b->st, &g);
        if (g) cudaGraphDestroy(g);
        b->cur = c0;
        throw;
    }
    ckb(cudaStreamEndCapture(b->st, &g), "capture");
    b->cur = c0;
    cudaGraphExec_t ge = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    ckb(e, "graph instantiate");
    b->graph[c0] = ge;
}

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace
}  // namespace flp

#define BATCH_TRY(...)                                           \
    try {                                                        \
        __VA_ARGS__;                                             \
        return FLP_OK;                                           \
    } catch (const flp::ConfigError& e) {                        \
        return flp::fail(FLP_ERR_INVALID_CONFIG, e.what());      \
    } catch (const std::invalid_argument& e) {                   \
        return flp::fail(FLP_ERR_INVALID_ARGUMENT, e.what());    \
    } catch (const flp::DeviceOom& e) {                          \
        return flp::fail(FLP_ERR_OOM, e.what());                 \
    } catch (const std::bad_alloc&) {                            \
        return flp::fail(FLP_ERR_OOM, "host allocation failed"); \
    } catch (const std::exception& e) {                          \
        return flp::fail(FLP_ERR_CUDA, e.what());                \
    }

#define BATCH_HANDLE(b) \
    if (!(b)) return flp::fail(FLP_ERR_INVALID_ARGUMENT, "null batch handle");

extern "C" {

int flp_batch_create(const char* const* config_jsons, int n_worlds, flp_batch** out) {
    if (!config_jsons || !out) return fail(FLP_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    flp_batch* b = new flp_batch();
    try {
        batch_create(b, config_jsons, n_worlds);
    } catch (...) {
        b->free_all();
        delete b;
        BATCH_TRY(throw)
    }
    *out = b;
    return FLP_OK;
}

int flp_batch_reconfigure(flp_batch* b, const char* const* config_jsons, int n_worlds) {
    BATCH_HANDLE(b);
    if (!config_jsons) return fail(FLP_ERR_INVALID_ARGUMENT, "null argument");
    BATCH_TRY(batch_reconfigure(b, config_jsons, n_worlds));
}

int flp_batch_destroy(flp_batch* b) {
    if (!b) return FLP_OK;
    cudaStreamSynchronize(b->st);
    b->free_all();
    delete b;
    return FLP_OK;
}

int flp_batch_write_world(flp_batch* b, int world, const float* state, size_t n) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (world < 0 || world >= b->n || !state) throw std::invalid_argument("bad world index or null state");
        const BWorld& d = b->hw[world];
        const size_t cn = size_t(d.C) * d.W * d.H;
        if (n != cn) throw std::invalid_argument("state size mismatch: expected " + std::to_string(cn));
        ckb(cudaMemcpyAsync(b->A[b->cur] + d.offA, state, cn * sizeof(float), cudaMemcpyHostToDevice, b->st), "copy");
        ckb(cudaStreamSynchronize(b->st), "sync");
        b->time[world] = 0.f;
        b->steps[world] = 0;
    })
}

int flp_batch_state_from_seed(flp_batch* b, int world, const char* seed_json) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (world < 0 || world >= b->n || !seed_json) throw std::invalid_argument("bad world index or null seed");
        std::vector<float> g = generate_seed(seed_json, b->cfgs[world]);
        const BWorld& d = b->hw[world];
        ckb(cudaMemcpyAsync(b->A[b->cur] + d.offA, g.data(), g.size() * sizeof(float), cudaMemcpyHostToDevice, b->st),
            "copy");
        ckb(cudaStreamSynchronize(b->st), "sync");
        b->time[world] = 0.f;
        b->steps[world] = 0;
    })
}

int flp_batch_states_from_seeds(flp_batch* b, const char* const* seed_jsons, int n) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (!seed_jsons || n != b->n) throw std::invalid_argument("need one seed entry per world");
        // generate on the host straight into one staging copy of the state pool
        // (left uninitialised: each seeded world fills its whole range); worlds
        // without a seed keep their device state, so copy runs of seeded worlds
        std::unique_ptr<float[]> staging(new float[std::max<size_t>(b->cells_total, 1)]);
        float* pool = staging.get();
        std::vector<char> seeded(n, 0);
        parallel_for(n, [&](int w) {  // worlds write disjoint ranges of the pool
            if (!seed_jsons[w]) return;
            generate_seed_into(seed_jsons[w], b->cfgs[w], pool + b->hw[w].offA);
            seeded[w] = 1;
        });
        for (int w = 0; w < n;) {
            if (!seeded[w]) { ++w; continue; }
            int e = w;
            while (e < n && seeded[e]) ++e;
            const long long off = b->hw[w].offA;
            const long long end = e < n ? b->hw[e].offA : (long long)b->cells_total;
            ckb(cudaMemcpyAsync(b->A[b->cur] + off, pool + off, size_t(end - off) * sizeof(float),
                                cudaMemcpyHostToDevice, b->st), "copy");
            w = e;
        }
        ckb(cudaStreamSynchronize(b->st), "sync");
        for (int w = 0; w < n; ++w)
            if (seeded[w]) {
                b->time[w] = 0.f;
                b->steps[w] = 0;
            }
    })
}

int flp_batch_read_world(flp_batch* b, int world, float* out, size_t n, float* time, uint64_t* step) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (world < 0 || world >= b->n || !out) throw std::invalid_argument("bad world index or null output");
        const BWorld& d = b->hw[world];
        const size_t cn = size_t(d.C) * d.W * d.H;
        if (n != cn) throw std::invalid_argument("state size mismatch: expected " + std::to_string(cn));
        ckb(cudaMemcpyAsync(out, b->A[b->cur] + d.offA, cn * sizeof(float), cudaMemcpyDeviceToHost, b->st), "copy");
        ckb(cudaStreamSynchronize(b->st), "sync");
        if (time) *time = b->time[world];
        if (step) *step = b->steps[world];
    })
}

int flp_batch_run(flp_batch* b, uint64_t n) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        while (n >= uint64_t(BATCH_GRAPH_STEPS)) {
            if (!b->graph[b->cur]) batch_build_graph(b);
            ckb(cudaGraphLaunch(b->graph[b->cur], b->st), "graph launch");
            b->advance(BATCH_GRAPH_STEPS);
            n -= BATCH_GRAPH_STEPS;
        }
        for (uint64_t i = 0; i < n; ++i) {
            b->enqueue_step();
            b->advance(1);
        }
    })
}

int flp_batch_synchronize(flp_batch* b) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        ckb(cudaStreamSynchronize(b->st), "sync");
        int status = 0;
        ckb(cudaMemcpy(&status, b->d_status, sizeof(int), cudaMemcpyDeviceToHost), "copy");
        if (status) {
            ckb(cudaMemset(b->d_status, 0, sizeof(int)), "memset");
            if (status & STATUS_NONFINITE) {
                g_last_error = "non-finite mass in a world";
                return FLP_ERR_NONFINITE;
            }
        }
    })
}

int flp_batch_synchronize_for(flp_batch* b, double timeout_ms) {
    BATCH_HANDLE(b);
    try {
        if (!wait_stream_for(b->st, timeout_ms))
            return fail(FLP_ERR_TIMEOUT, "the batch's stream did not finish within " + std::to_string(timeout_ms) + " ms");
    } catch (const std::exception& e) {
        return fail(FLP_ERR_CUDA, e.what());
    }
    return flp_batch_synchronize(b);
}

int flp_batch_total_mass(flp_batch* b, double* per_world, int n) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (!per_world || n != b->n) throw std::invalid_argument("output needs one double per world");
        k_batch_mass<<<b->n, 256, 0, b->st>>>(b->d_worlds, b->A[b->cur], b->d_mass);
        ckb(cudaGetLastError(), "mass");
        ckb(cudaMemcpyAsync(per_world, b->d_mass, n * sizeof(double), cudaMemcpyDeviceToHost, b->st), "copy");
        ckb(cudaStreamSynchronize(b->st), "sync");
    })
}

int flp_batch_stats(flp_batch* b, double* out, size_t n) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (!out || n != size_t(b->n) * FLP_BATCH_NSTAT)
            throw std::invalid_argument("output needs FLP_BATCH_NSTAT doubles per world");
        k_batch_stats<<<b->n, 256, 0, b->st>>>(b->d_worlds, b->A[b->cur], b->d_stats);
        ckb(cudaGetLastError(), "stats");
        ckb(cudaMemcpyAsync(out, b->d_stats, n * sizeof(double), cudaMemcpyDeviceToHost, b->st), "copy");
        ckb(cudaStreamSynchronize(b->st), "sync");
    })
}

int flp_batch_reserve_snapshots(flp_batch* b, int n_slots) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (n_slots < 0) throw std::invalid_argument("negative slot count");
        if (n_slots <= b->n_snap) return FLP_OK;
        ckb(cudaStreamSynchronize(b->st), "sync");
        if (b->d_snaps) flp::dfree(b->d_snaps);
        b->d_snaps = nullptr;
        b->n_snap = 0;
        b->d_snaps = dalloc_b<float>(size_t(n_slots) * b->cells);
        b->n_snap = n_slots;
    })
}

int flp_batch_snapshot(flp_batch* b, int slot) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (slot < 0 || slot >= b->n_snap) throw std::invalid_argument("snapshot slot out of range");
        k_batch_snapshot<<<b->n, 256, 0, b->st>>>(b->d_worlds, b->A[b->cur], b->d_celloff, b->d_snaps, b->cells,
                                                  slot);
        ckb(cudaGetLastError(), "snapshot");
    })
}

int flp_batch_similarity(flp_batch* b, int slot_a, int slot_b, double* out, int n) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (slot_a < 0 || slot_b < 0 || slot_a >= b->n_snap || slot_b >= b->n_snap)
            throw std::invalid_argument("snapshot slot out of range");
        if (!out || n != b->n) throw std::invalid_argument("output needs one double per world");
        k_batch_similarity<<<b->n, 256, 0, b->st>>>(b->d_worlds, b->d_celloff, b->d_snaps, b->cells, slot_a, slot_b,
                                                    b->d_stats);
        ckb(cudaGetLastError(), "similarity");
        ckb(cudaMemcpyAsync(out, b->d_stats, n * sizeof(double), cudaMemcpyDeviceToHost, b->st), "copy");
        ckb(cudaStreamSynchronize(b->st), "sync");
    })
}

int flp_batch_kernel_spectra(flp_batch* b, int* unique_sets, size_t* bytes) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (unique_sets) *unique_sets = b->unique_spectra;
        if (bytes) *bytes = b->kh_bytes;
    })
}

int flp_batch_info(flp_batch* b, int* n_worlds, size_t* cell_channels, size_t* cells) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (n_worlds) *n_worlds = b->n;
        if (cell_channels) *cell_channels = b->cells_total;
        if (cells) {
            size_t s = 0;
            for (const auto& d : b->hw) s += size_t(d.W) * d.H;
            *cells = s;
        }
    })
}

void* flp_batch_stream(flp_batch* b) { return b ? static_cast<void*>(b->st) : nullptr; }

int flp_batch_profile_run(flp_batch* b, int steps, int flush_l2, float* stage_ms, float* step_ms) {
    BATCH_HANDLE(b);
    BATCH_TRY({
        if (steps < 0) throw std::invalid_argument("negative step count");
        if (flush_l2 && !b->flush_buf) {
            int dev = 0, l2 = 0;
            ckb(cudaGetDevice(&dev), "device");
            ckb(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev), "attr");
            b->flush_bytes = std::max<size_t>(size_t(2) * size_t(l2), size_t(64) << 20);
            ckb(flp::dmalloc(&b->flush_buf, b->flush_bytes), "flush buffer");
        }
        // Up to RING steps in flight, each with its own events, so the host
        // enqueues ahead of the device; without stage_ms only whole steps are
        // bracketed.
        constexpr int RING = 16, E = NSTAGE + 1;
        while (int(b->pev.size()) < RING * E) {
            cudaEvent_t e;
            ckb(cudaEventCreate(&e), "event");
            b->pev.push_back(e);
        }
        const bool staged = stage_ms != nullptr;
        double acc[NSTAGE] = {0}, tot = 0;
        auto harvest = [&](int slot) {
            cudaEvent_t* ev = b->pev.data() + size_t(slot) * E;
            ckb(cudaEventSynchronize(ev[NSTAGE]), "sync");
            for (int i = 0; staged && i < NSTAGE; ++i) {
                float ms = 0.f;
                ckb(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]), "elapsed");
                acc[i] += ms;
            }
            float ms = 0.f;
            ckb(cudaEventElapsedTime(&ms, ev[0], ev[NSTAGE]), "elapsed");
            tot += ms;
        };
        for (int s = 0; s < steps; ++s) {
            const int slot = s % RING;
            if (s >= RING) harvest(slot);
            if (flush_l2) ckb(cudaMemsetAsync(b->flush_buf, s & 0xFF, b->flush_bytes, b->st), "flush");
            b->enqueue_step(b->pev.data() + size_t(slot) * E, staged);
            b->advance(1);
        }
        for (int s = std::max(0, steps - RING); s < steps; ++s) harvest(s % RING);
        if (stage_ms)
            for (int i = 0; i < NSTAGE; ++i) stage_ms[i] = float(acc[i]);
        if (step_ms) *step_ms = float(tot);
    })
}

}  // extern "C"
