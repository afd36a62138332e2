// Host runtime of the engine and its C ABI (include/flowlenia_cuda.h).
//
// One flp_propagator owns a CUDA stream and all device buffers of one world:
// the state (double-buffered; the reference swaps `channels` with
// `next_channels`, src/compute/propagator.rs:416-419), the affinity field,
// the convolution scratch (kernel spectra or stencil taps) and two flow-bound
// slots that follow the state buffers.  A step is 2 kernels on the direct
// path or 4 on the FFT path; run(n) replays a captured CUDA graph of
// GRAPH_STEPS steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "device_mem.h"
#include "flowlenia_cuda.h"
#include "kernels.h"
#include "schema.h"

namespace flp {

thread_local std::string g_last_error;

// Steps per captured CUDA graph (even, so a replay leaves the state in the
// buffer it started from).
constexpr int GRAPH_STEPS = 16;

struct FlpError : std::runtime_error {
    int code;
    FlpError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        int code = (e == cudaErrorMemoryAllocation) ? FLP_ERR_OOM : FLP_ERR_CUDA;
        throw FlpError(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
#define CK(x) cuda_check((x), #x)

template <class T>
T* dalloc(size_t n) {
    if (n == 0) n = 1;
    void* p = nullptr;
    CK(flp::dmalloc(&p, n * sizeof(T)));
    return static_cast<T*>(p);
}

bool make_plan(int L, FftPlan& p) {
    p = FftPlan();
    p.L = L;
    int m = L;
    const int rads[4] = {4, 2, 3, 5};
    for (int r : rads)
        while (m % r == 0 && p.nst < 24) {
            p.rad[p.nst++] = r;
            m /= r;
        }
    return m == 1 && L >= 1;
}

static void upload_twiddles(std::vector<float2>& dst, int L, int count) {
    for (int t = 0; t < count; ++t) {
        double ang = -2.0 * M_PI * double(t) / double(L);
        dst.push_back(make_float2(float(std::cos(ang)), float(std::sin(ang))));
    }
}

static std::once_flag g_attr_once;
static void set_attributes_once() {
    std::call_once(g_attr_once, [] {
        transport_2d_set_attributes();
        transport_3d_set_attributes();
        fft2d_set_attributes(200 * 1024);
        fft3d_set_attributes(200 * 1024);
    });
}

// Measured launch choices of one world shape, cached per (W, H, D, channels,
// kernels, largest kernel radius, source channels) for the process.  Every
// choice gives the same bits: only the time differs.
struct Tuning {
    int conv_mode = -1;                                    // FLP_CONV_DIRECT / FLP_CONV_FFT; -1 = not measured
    int wpc_r2c = 8, wpc_cols = 8, share_cols = 1, wpc_c2r = 8;  // FFT passes (FftGeom)
    int gather_gby = 1;                                    // destination rows per gather thread (1 or 2)
    bool fft_tuned = false, gather_tuned = false;
};
static std::mutex g_tune_mu;
static std::map<std::vector<int>, Tuning> g_tune_cache;

}  // namespace flp

using namespace flp;

struct flp_propagator {
    SimulationConfig cfg;
    int W = 0, H = 0, D = 1, C = 0, K = 0, dims = 2;
    size_t N = 0;
    cudaStream_t st = nullptr;
    float* A[2] = {nullptr, nullptr};
    int cur = 0;
    float* U = nullptr;
    std::vector<KDesc> kd;
    KDesc* d_kd = nullptr;
    float* d_taps = nullptr;
    int rmax = 0;
    bool direct_ok = false;
    FlowParams fp{};
    int* d_dmax = nullptr;   // largest |dest - x| of the step (float bits), reset by the step's first kernel
    float* d_DX = nullptr;   // per-channel destinations (C x N each)
    float* d_DY = nullptr;
    float* d_DZ = nullptr;   // 3D only
    int* d_status = nullptr;
    double2* d_partial = nullptr;
    double* d_mass = nullptr;
    int np = 0;
    // FFT path
    bool fft_ok = false;
    FftGeom geom;
    float2* d_tw = nullptr;
    float2* d_S = nullptr;
    float2* d_T = nullptr;
    float2* d_KH = nullptr;
    int* d_srcs = nullptr;
    int* d_slot = nullptr;
    int nsrc = 0;
    std::vector<int> h_srcs;  // the source channels, in slot order
    int conv_mode = FLP_CONV_DIRECT;
    bool conv_pending = true;  // the autotuner runs before the first convolution unless a mode is set first
    int gather_gby = 1;        // destination rows per gather thread
    bool tuning_cached = false;  // the last tuning came from the process cache
    float time = 0.f;
    uint64_t step = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t graph1[2] = {nullptr, nullptr};  // one step from A[cur] to A[cur ^ 1]
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // profiling
    std::vector<cudaEvent_t> prof_ev;
    int prof_base = 0;  // first event of the step being recorded
    void* flush_buf = nullptr;
    size_t flush_bytes = 0;

    // Stage hook: called after each kernel of a step with its stage index
    // (used by flp_profile_run to record events between kernels).
    using Hook = void (*)(flp_propagator*, int);
    Hook hook = nullptr;
    void mark(int stage) {
        if (hook) hook(this, stage);
    }

    // hin (2D FFT path only, see host_io_ok): the source planes are read from
    // there (mapped host memory) and left behind in a.
    void enqueue_conv(const float* a, int* reset_slot, const float* hin = nullptr) {
        if (K == 0) {
            // No kernels: the affinity stays zero (it is cleared at creation).
            launch_zero_ints(reset_slot, 1, st);
            mark(0);
            return;
        }
        if (dims == 3) {
            // x rows are the D*H rows of the grid; spectra are [kx][z][y]
            const int Wc = W / 2 + 1;
            launch_fft_r2c(a, d_S, d_srcs, nsrc, W, D * H, geom, reset_slot, 1, st);
            mark(0);
            launch_fft_lines(d_S, nullptr, d_S, nullptr, nsrc, Wc * D, H, geom, 1, 1.f, st);
            mark(1);
            launch_fft_z(d_S, d_KH, d_T, d_slot, K, W, H, D, geom.twD, 0, 1.f, st);
            mark(2);
            launch_fft_lines(d_T, nullptr, d_T, nullptr, K, Wc * D, H, geom, 2, 1.f, st);
            mark(3);
            launch_fft_c2r_growth(d_T, U, d_kd, K, W, D * H, C, geom, st);
            mark(4);
        } else if (conv_mode == FLP_CONV_DIRECT) {
            launch_conv_direct_2d(a, U, d_kd, K, d_taps, W, H, C, rmax, reset_slot, st);
            mark(0);
        } else {
            if (hin) launch_fft_r2c(hin, d_S, d_srcs, nsrc, W, H, geom, reset_slot, 1, st, const_cast<float*>(a));
            else launch_fft_r2c(a, d_S, d_srcs, nsrc, W, H, geom, reset_slot, 1, st);
            mark(0);
            launch_fft_cols_conv(d_S, d_KH, d_T, d_slot, nsrc, K, 1, W, H, geom, st);
            mark(1);
            launch_fft_c2r_growth(d_T, U, d_kd, K, W, H, C, geom, st);
            mark(2);
        }
    }

    std::vector<std::string> stage_names() const {
        if (dims == 3) {
            if (K == 0) return {"slot_reset", "flow_3d", "gather_3d"};
            return {"fft_x_r2c", "fft_y_fwd", "fft_z_conv", "fft_y_inv", "fft_x_c2r_growth", "flow_3d", "gather_3d"};
        }
        if (K == 0) return {"slot_reset", "flow_2d", "gather_2d"};
        if (conv_mode == FLP_CONV_DIRECT) return {"conv_direct_growth_2d", "flow_2d", "gather_2d"};
        return {"fft_rows_r2c", "fft_cols_conv", "fft_rows_c2r_growth", "flow_2d", "gather_2d"};
    }

    void enqueue_transport(const float* a, float* an) {
        const int ns = int(stage_names().size());
        if (dims == 3) {
            launch_flow_3d(a, U, d_DX, d_DY, d_DZ, C, W, H, D, fp, d_dmax, d_status, st);
            mark(ns - 2);
            launch_gather_3d(d_DX, d_DY, d_DZ, a, an, C, W, H, D, fp, d_dmax, st);
            mark(ns - 1);
            return;
        }
        launch_flow_2d(a, U, d_DX, d_DY, C, W, H, fp, d_dmax, d_status, st);
        mark(ns - 2);
        launch_gather_2d(d_DX, d_DY, a, an, C, W, H, fp, d_dmax, gather_gby, st);
        mark(ns - 1);
    }

    void enqueue_step(const float* hin = nullptr) {
        const float* a = A[cur];
        float* an = A[cur ^ 1];
        enqueue_conv(a, d_dmax, hin);
        enqueue_transport(a, an);
        CK(cudaGetLastError());
        cur ^= 1;
    }

    // Whether a host-state call may read a device-addressable host buffer from
    // the step's own kernels: 2D, FFT convolution, and a width whose row
    // transform has the copy-through form.
    bool host_io_ok() const {
        return dims == 2 && K > 0 && conv_mode == FLP_CONV_FFT && fft_rows_copy_width(W);
    }

    void advance_clock(uint64_t n) {
        for (uint64_t i = 0; i < n; ++i) time += cfg.dt;  // f32 accumulation, propagator.rs:418
        step += n;
    }

    void free_all() {
        for (auto& g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        for (auto& g : graph1)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        void* ptrs[] = {A[0], A[1], U, d_kd, d_taps, d_dmax, d_DX, d_DY, d_DZ, d_status, d_partial, d_mass,
                        d_tw, d_S, d_T, d_KH, d_srcs, d_slot};
        for (void* p : ptrs)
            if (p) flp::dfree(p);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto e : prof_ev) cudaEventDestroy(e);
        if (flush_buf) flp::dfree(flush_buf);
        if (st) cudaStreamDestroy(st);
    }
};

namespace flp {

static void setup_direct(flp_propagator* h, const std::vector<KernelStencil>& ks) {
    // Taps: flipped effective stencil (convolution, not correlation); when
    // 2r+1 exceeds a side, offsets that alias onto one torus cell keep a
    // single tap carrying the wrap-padded value (kernel.rs:98-117).
    std::vector<float> taps;
    h->rmax = 0;
    for (int k = 0; k < h->K; ++k) {
        const KernelStencil& s = ks[k];
        int r = s.radius, side = s.size;
        h->rmax = std::max(h->rmax, r);
        h->kd[k].r = r;
        h->kd[k].tap_off = int(taps.size());
        std::vector<float> pad = pad_kernel(s, h->W, h->H, 1);
        std::vector<float> eff(size_t(side) * side, 0.f);
        std::vector<char> seen(size_t(h->W) * h->H, 0);
        for (int dy = -r; dy <= r; ++dy)
            for (int dx = -r; dx <= r; ++dx) {
                int tx = ((dx % h->W) + h->W) % h->W, ty = ((dy % h->H) + h->H) % h->H;
                size_t t = size_t(ty) * h->W + tx;
                if (seen[t]) continue;
                seen[t] = 1;
                // out[x] = sum_d A[x - d] S[d] = sum_d A[x + d] S[-d]
                eff[size_t(-dy + r) * side + (-dx + r)] = pad[t];
            }
        taps.insert(taps.end(), eff.begin(), eff.end());
    }
    h->direct_ok = h->rmax <= MAX_DIRECT_RADIUS;
    if (!taps.empty()) {
        h->d_taps = dalloc<float>(taps.size());
        CK(cudaMemcpy(h->d_taps, taps.data(), taps.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
}

static void setup_fft(flp_propagator* h, const std::vector<KernelStencil>& ks) {
    const int W = h->W, H = h->H;
    h->fft_ok = false;
    if (W % 2 != 0 || W < 2) return;
    FftGeom g;
    if (!make_plan(W / 2, g.pm) || !make_plan(H, g.ph)) return;
    const int M = W / 2, Wc = M + 1;
    g.NR = 8;
    while (g.NR > 1 && fft_rows_smem(W, g.NR, true) > 200 * 1024) g.NR /= 2;
    g.NC = 8;
    while (g.NC > 1 && fft_cols_smem(H, g.NC) > 200 * 1024) g.NC /= 2;
    if (fft_rows_smem(W, g.NR, true) > 200 * 1024 || fft_cols_smem(H, g.NC) > 200 * 1024) return;
    std::vector<float2> tw;
    upload_twiddles(tw, M, M);
    upload_twiddles(tw, W, Wc);
    upload_twiddles(tw, H, H);
    h->d_tw = dalloc<float2>(tw.size());
    CK(cudaMemcpy(h->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice));
    g.twM = h->d_tw;
    g.twW = h->d_tw + M;
    g.twH = h->d_tw + M + Wc;
    h->geom = g;
    // source channels and their spectrum slots
    std::vector<int> srcs, slot(h->K);
    for (int k = 0; k < h->K; ++k) {
        auto it = std::find(srcs.begin(), srcs.end(), h->kd[k].src);
        if (it == srcs.end()) { slot[k] = int(srcs.size()); srcs.push_back(h->kd[k].src); }
        else slot[k] = int(it - srcs.begin());
    }
    h->nsrc = int(srcs.size());
    h->h_srcs = srcs;
    h->d_srcs = dalloc<int>(srcs.size());
    h->d_slot = dalloc<int>(slot.size());
    CK(cudaMemcpy(h->d_srcs, srcs.data(), srcs.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_slot, slot.data(), slot.size() * sizeof(int), cudaMemcpyHostToDevice));
    const size_t spec = size_t(Wc) * H;
    h->d_S = dalloc<float2>(spec * std::max(h->nsrc, 1));
    h->d_T = dalloc<float2>(spec * h->K);
    h->d_KH = dalloc<float2>(spec * h->K);
    // Kernel spectra: FFT of the wrap-padded stencils, scaled by 1/(W*H)
    // (the inverse's normalisation, fft.rs:389, folded in once).
    std::vector<float> padded(size_t(h->K) * W * H);
    for (int k = 0; k < h->K; ++k) {
        std::vector<float> p = pad_kernel(ks[k], W, H, 1);
        std::copy(p.begin(), p.end(), padded.begin() + size_t(k) * W * H);
    }
    DevScratch scratch;
    float* d_pad = scratch.add(dalloc<float>(padded.size()));
    float2* d_tmp = scratch.add(dalloc<float2>(spec * h->K));
    CK(cudaMemcpyAsync(d_pad, padded.data(), padded.size() * sizeof(float), cudaMemcpyHostToDevice, h->st));
    launch_fft_r2c(d_pad, d_tmp, nullptr, h->K, W, H, g, nullptr, 0, h->st);
    launch_fft_cols(d_tmp, nullptr, h->d_KH, nullptr, h->K, W, H, g, 1, float(1.0 / (double(W) * double(H))), h->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->st));
    h->fft_ok = true;
}

static void setup_fft3d(flp_propagator* h, const std::vector<KernelStencil>& ks) {
    const int W = h->W, H = h->H, D = h->D;
    h->fft_ok = false;
    if (W % 2 != 0 || !fft_row_templated(W / 2) || !fft_col_templated(H) || !fft_z_templated(D))
        throw FlpError(FLP_ERR_UNSUPPORTED,
                       "3D worlds need an even width with W/2 in {16..256}, H in {32..512}, D in {32..256} (factors 2, 3)");
    if (h->C > flow3d_max_channels())
        throw FlpError(FLP_ERR_UNSUPPORTED,
                       "3D worlds support at most " + std::to_string(flow3d_max_channels()) + " channels");
    FftGeom g;
    make_plan(W / 2, g.pm);
    make_plan(H, g.ph);
    const int M = W / 2, Wc = M + 1;
    std::vector<float2> tw;
    upload_twiddles(tw, M, M);
    upload_twiddles(tw, W, Wc);
    upload_twiddles(tw, H, H);
    upload_twiddles(tw, D, D);
    h->d_tw = dalloc<float2>(tw.size());
    CK(cudaMemcpy(h->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice));
    g.twM = h->d_tw;
    g.twW = h->d_tw + M;
    g.twH = h->d_tw + M + Wc;
    g.twD = h->d_tw + M + Wc + H;
    h->geom = g;
    std::vector<int> srcs, slot(h->K);
    for (int k = 0; k < h->K; ++k) {
        auto it = std::find(srcs.begin(), srcs.end(), h->kd[k].src);
        if (it == srcs.end()) { slot[k] = int(srcs.size()); srcs.push_back(h->kd[k].src); }
        else slot[k] = int(it - srcs.begin());
    }
    h->nsrc = int(srcs.size());
    h->d_srcs = dalloc<int>(srcs.size());
    h->d_slot = dalloc<int>(slot.size());
    if (!srcs.empty()) CK(cudaMemcpy(h->d_srcs, srcs.data(), srcs.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (!slot.empty()) CK(cudaMemcpy(h->d_slot, slot.data(), slot.size() * sizeof(int), cudaMemcpyHostToDevice));
    const size_t spec = size_t(Wc) * H * D;
    h->d_S = dalloc<float2>(spec * std::max(h->nsrc, 1));
    h->d_T = dalloc<float2>(spec * std::max(h->K, 1));
    h->d_KH = dalloc<float2>(spec * std::max(h->K, 1));
    if (h->K) {
        // K^ = FFT3(wrap-padded stencil) / (W*H*D), in the [kx][z][y] layout
        std::vector<float> padded(size_t(h->K) * W * H * D);
        for (int k = 0; k < h->K; ++k) {
            std::vector<float> p = pad_kernel(ks[k], W, H, D);
            std::copy(p.begin(), p.end(), padded.begin() + size_t(k) * W * H * D);
        }
        DevScratch scratch;
        float* d_pad = scratch.add(dalloc<float>(padded.size()));
        float2* d_tmp = scratch.add(dalloc<float2>(spec * h->K));
        CK(cudaMemcpyAsync(d_pad, padded.data(), padded.size() * sizeof(float), cudaMemcpyHostToDevice, h->st));
        launch_fft_r2c(d_pad, d_tmp, nullptr, h->K, W, D * H, g, nullptr, 0, h->st);
        launch_fft_lines(d_tmp, nullptr, d_tmp, nullptr, h->K, Wc * D, H, g, 1, 1.f, h->st);
        launch_fft_z(d_tmp, nullptr, h->d_KH, nullptr, h->K, W, H, D, g.twD, 1,
                     float(1.0 / (double(W) * double(H) * double(D))), h->st);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->st));
    }
    h->fft_ok = true;
}

// The tuner's stopwatch: every timed repetition starts with the L2 cache
// flushed (a memset of twice its size, outside the timed interval), so the
// candidates are ranked as they run when a step's inputs come from HBM: every
// world or batch larger than L2, and every step measured after a flush.  (For
// a world small enough to stay in L2 across back-to-back steps, the warm
// ranking differs by about 1 us at 512x512: the flushed step there favours one
// destination row per gather thread and 4-warp column CTAs, the warm one two
// rows and 8 warps.)
struct ColdTimer {
    static constexpr int MAX_REPS = 20;
    flp_propagator* h;
    DevScratch scratch;
    void* flush = nullptr;
    size_t bytes = 0;
    cudaEvent_t ev[2 * MAX_REPS] = {};
    explicit ColdTimer(flp_propagator* hh) : h(hh) {
        int dev = 0, l2 = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
        bytes = std::max<size_t>(size_t(2) * size_t(l2), size_t(64) << 20);
        flush = scratch.add(dalloc<char>(bytes));
        for (auto& e : ev) CK(cudaEventCreate(&e));
    }
    ~ColdTimer() {
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    }
    ColdTimer(const ColdTimer&) = delete;
    ColdTimer& operator=(const ColdTimer&) = delete;
    // Mean device time of enqueue() over reps flushed repetitions, after two
    // untimed ones.
    template <class F>
    float time(F&& enqueue, int reps) {
        reps = std::min(reps, MAX_REPS);
        enqueue();
        enqueue();
        for (int i = 0; i < reps; ++i) {
            CK(cudaMemsetAsync(flush, i & 0xFF, bytes, h->st));
            CK(cudaEventRecord(ev[2 * i], h->st));
            enqueue();
            CK(cudaEventRecord(ev[2 * i + 1], h->st));
        }
        CK(cudaEventSynchronize(ev[2 * reps - 1]));
        float total = 0.f;
        for (int i = 0; i < reps; ++i) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]));
            total += ms;
        }
        return total / reps;
    }
};

static float time_conv(flp_propagator* h, ColdTimer& tm, int mode, int reps) {
    int saved = h->conv_mode;
    h->conv_mode = mode;
    const float ms = tm.time([&] { h->enqueue_conv(h->A[h->cur], nullptr); }, reps);
    h->conv_mode = saved;
    return ms;
}

// Device time of one full step (from A[cur] into the other buffer, which is
// scratch until the next step).
static float time_step(flp_propagator* h, ColdTimer& tm, int reps) {
    const float* a = h->A[h->cur];
    float* an = h->A[h->cur ^ 1];
    return tm.time([&] {
        h->enqueue_conv(a, h->d_dmax);
        h->enqueue_transport(a, an);
    }, reps);
}

static void apply_tuning(flp_propagator* h, const Tuning& t) {
    h->geom.wpc_r2c = t.wpc_r2c;
    h->geom.wpc_cols = t.wpc_cols;
    h->geom.share_cols = t.share_cols;
    h->geom.wpc_c2r = t.wpc_c2r;
    h->gather_gby = t.gather_gby;
}

// Each FFT pass's CTA shape (warps per CTA; for the columns also one forward
// transform per source or per kernel), one pass at a time from the defaults,
// each candidate timed over 20 whole convolutions.
static void tune_fft_passes(flp_propagator* h, ColdTimer& tm, Tuning& t) {
    const int reps = 20;
    auto timed = [&](const Tuning& c) {
        apply_tuning(h, c);
        return time_conv(h, tm, FLP_CONV_FFT, reps);
    };
    float best = timed(t);
    for (int w : {4}) {
        Tuning c = t;
        c.wpc_r2c = w;
        const float ms = timed(c);
        if (ms < best) { best = ms; t = c; }
    }
    for (int share : {1, 0})
        for (int w : {8, 4}) {
            if (share == t.share_cols && w == t.wpc_cols) continue;
            Tuning c = t;
            c.share_cols = share;
            c.wpc_cols = w;
            const float ms = timed(c);
            if (ms < best) { best = ms; t = c; }
        }
    {
        Tuning c = t;
        c.wpc_c2r = 4;
        const float ms = timed(c);
        if (ms < best) { best = ms; t = c; }
    }
    apply_tuning(h, t);
}

// Destination rows per gather thread, timed over whole steps.
static void tune_gather(flp_propagator* h, ColdTimer& tm, Tuning& t) {
    float best = 0.f;
    int pick = 1;
    for (int gby : {1, 2}) {
        h->gather_gby = gby;
        const float ms = time_step(h, tm, 10);
        if (gby == 1 || ms < best) { best = ms; pick = gby; }
    }
    t.gather_gby = pick;
    h->gather_gby = pick;
}

static void resolve_conv_mode(flp_propagator* h, int requested) {
    if (h->K == 0) { h->conv_mode = FLP_CONV_DIRECT; return; }
    if (requested == FLP_CONV_DIRECT && !h->direct_ok)
        throw FlpError(FLP_ERR_UNSUPPORTED, "direct convolution supports radius <= 24");
    if (requested == FLP_CONV_FFT && !h->fft_ok)
        throw FlpError(FLP_ERR_UNSUPPORTED, "FFT path needs an even width and sides of factors 2,3,5");
    if (!h->fft_ok && !h->direct_ok)
        throw FlpError(FLP_ERR_UNSUPPORTED, "no convolution path for this grid/radius");
    const std::vector<int> key = {h->W, h->H, h->D, h->C, h->K, h->rmax, h->nsrc};
    Tuning t;
    bool cached = false;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            t = it->second;
            cached = true;
        }
    }
    bool measured = false;
    std::unique_ptr<ColdTimer> tm;
    auto timer = [&]() -> ColdTimer& {
        if (!tm) tm.reset(new ColdTimer(h));
        return *tm;
    };
    int mode;
    if (requested == FLP_CONV_DIRECT || requested == FLP_CONV_FFT) mode = requested;
    else if (!h->fft_ok) mode = FLP_CONV_DIRECT;
    else if (!h->direct_ok) mode = FLP_CONV_FFT;
    else if (t.conv_mode >= 0) mode = t.conv_mode;
    else {
        apply_tuning(h, t);
        const float t_direct = time_conv(h, timer(), FLP_CONV_DIRECT, 5);
        const float t_fft = time_conv(h, timer(), FLP_CONV_FFT, 5);
        mode = t.conv_mode = t_fft < t_direct ? FLP_CONV_FFT : FLP_CONV_DIRECT;
        measured = true;
    }
    h->conv_mode = mode;
    apply_tuning(h, t);
    if (h->dims == 2 && mode == FLP_CONV_FFT && !t.fft_tuned && fft_row_templated(h->W / 2) &&
        fft_col_templated(h->H)) {
        tune_fft_passes(h, timer(), t);
        t.fft_tuned = measured = true;
    }
    if (h->dims == 2 && !t.gather_tuned) {
        tune_gather(h, timer(), t);
        t.gather_tuned = measured = true;
    }
    h->tuning_cached = cached && !measured;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = t;
}

PropView prop_view(flp_propagator* h) {
    PropView v{};
    v.state = h->A[h->cur];
    v.stream = h->st;
    v.width = h->W;
    v.height = h->H;
    v.depth = h->D;
    v.channels = h->C;
    v.dt = h->cfg.dt;
    cudaGetDevice(&v.device);
    return v;
}

FlowParams flow_params_of(const SimulationConfig& cfg) {
    FlowParams fp{};
    fp.dt = cfg.dt;
    fp.s = cfg.flow.distribution_size;
    // Square area (2s)^2 in 2D (reintegration.rs:117); cube volume (2s)^3 in
    // 3D (reintegration3d.rs:137), both evaluated left to right in f32.
    float two_s = 2.0f * fp.s;
    fp.total_area = two_s * two_s;
    if (cfg.is_3d()) fp.total_area = fp.total_area * two_s;
    int e = 0;
    float mant = std::frexp(fp.total_area, &e);
    fp.area_pow2 = (fp.total_area > 0.f && mant == 0.5f && std::isnormal(fp.total_area)) ? 1 : 0;
    fp.inv_area = fp.area_pow2 ? 1.0f / fp.total_area : 0.f;
    fp.beta_a = cfg.flow.beta_a;
    {
        int eb = 0;
        const float mb = std::frexp(fp.beta_a, &eb);
        fp.beta_pow2 = (fp.beta_a > 0.f && mb == 0.5f && std::isnormal(fp.beta_a) && std::isnormal(1.0f / fp.beta_a)) ? 1 : 0;
        fp.inv_beta = fp.beta_pow2 ? 1.0f / fp.beta_a : 0.f;
    }
    fp.nexp = cfg.flow.n;
    fp.point_mode = fp.total_area < 1e-10f ? 1 : 0;
    if (fp.point_mode) fp.area_pow2 = 0;  // nearest-cell deposits carry the raw mass
    // With 2s >= 1.5 no rounded square [dest - s, dest + s] fits inside one cell,
    // which the 2D gather's saturating overlap form relies on.
    fp.wide_square = fp.area_pow2 && fp.s >= 0.75f ? 1 : 0;
    // dest = x + dt*F and x_min/x_max are rounded at the scale of the largest
    // coordinate; allow a few ulps of it plus a fixed slack.
    const float maxside = float(std::max(std::max(cfg.width, cfg.height), cfg.depth));
    fp.pos_eps = 8.0f * maxside * 1.1920929e-07f + 1e-4f;
    return fp;
}

static void create(const std::string& json, flp_propagator* h) {
    h->cfg = parse_config(json);
    const SimulationConfig& c = h->cfg;
    h->W = c.width; h->H = c.height; h->D = c.depth; h->C = c.channels; h->K = int(c.kernels.size());
    h->dims = c.is_3d() ? 3 : 2;
    h->N = c.grid_size();
    set_attributes_once();
    CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    const size_t CN = size_t(h->C) * h->N;
    h->A[0] = dalloc<float>(CN);
    h->A[1] = dalloc<float>(CN);
    h->U = dalloc<float>(CN);
    CK(cudaMemsetAsync(h->A[0], 0, CN * sizeof(float), h->st));
    CK(cudaMemsetAsync(h->A[1], 0, CN * sizeof(float), h->st));
    CK(cudaMemsetAsync(h->U, 0, CN * sizeof(float), h->st));
    h->d_dmax = dalloc<int>(1);
    h->d_DX = dalloc<float>(CN);
    h->d_DY = dalloc<float>(CN);
    if (h->dims == 3) h->d_DZ = dalloc<float>(CN);
    h->d_status = dalloc<int>(1);
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->st));
    h->np = 256;
    h->d_partial = dalloc<double2>(h->np);
    h->d_mass = dalloc<double>(1);
    // kernels
    std::vector<KernelStencil> ks;
    h->kd.resize(h->K);
    for (int k = 0; k < h->K; ++k) {
        const KernelConfig& kc = c.kernels[k];
        ks.push_back(build_kernel(kc, c.kernel_radius, h->dims));
        KDesc d{};
        d.src = kc.source_channel;
        d.tgt = kc.target_channel;
        d.weight = kc.weight;
        d.mu = kc.mu;
        float sigma_sq_2 = 2.0f * kc.sigma * kc.sigma;
        d.inv2s2 = 1.0f / sigma_sq_2;
        h->kd[k] = d;
    }
    if (h->dims == 2) {
        setup_direct(h, ks);
    } else {
        for (int k = 0; k < h->K; ++k) h->kd[k].r = ks[k].radius;
        h->direct_ok = false;  // 3D convolves through the FFT path only
    }
    h->d_kd = dalloc<KDesc>(h->kd.size());
    if (h->K) CK(cudaMemcpy(h->d_kd, h->kd.data(), h->kd.size() * sizeof(KDesc), cudaMemcpyHostToDevice));
    if (h->dims == 2) setup_fft(h, ks);
    else setup_fft3d(h, ks);
    h->fp = flow_params_of(c);
    CK(cudaStreamSynchronize(h->st));
    h->conv_pending = true;
}

// Runs the direct-vs-FFT autotuner on first use, outside any graph capture.
static void ensure_conv_mode(flp_propagator* h) {
    if (!h->conv_pending) return;
    resolve_conv_mode(h, FLP_CONV_AUTO);
    h->conv_pending = false;
}

static void upload_state(flp_propagator* h, const float* src, size_t n) {
    const size_t CN = size_t(h->C) * h->N;
    if (n != CN) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "state size mismatch: expected " + std::to_string(CN));
    CK(cudaMemcpyAsync(h->A[h->cur], src, CN * sizeof(float), cudaMemcpyHostToDevice, h->st));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->st));
}

static void build_graph(flp_propagator* h) {
    int c0 = h->cur;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    try {
        for (int i = 0; i < GRAPH_STEPS; ++i) h->enqueue_step();
    } catch (...) {
        cudaStreamEndCapture(h->st, &g);
        if (g) cudaGraphDestroy(g);
        h->cur = c0;
        throw;
    }
    CK(cudaStreamEndCapture(h->st, &g));
    h->cur = c0;  // GRAPH_STEPS is even: the graph leaves the state in the same buffer
    cudaGraphExec_t ge = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    h->graph[c0] = ge;
}

// A one-step graph per buffer parity, for the steps left over after the
// GRAPH_STEPS graphs (one launch instead of one per kernel).
static void build_graph1(flp_propagator* h) {
    const int c0 = h->cur;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    try {
        h->enqueue_step();
    } catch (...) {
        cudaStreamEndCapture(h->st, &g);
        if (g) cudaGraphDestroy(g);
        h->cur = c0;
        throw;
    }
    CK(cudaStreamEndCapture(h->st, &g));
    h->cur = c0;
    cudaGraphExec_t ge = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    h->graph1[c0] = ge;
}

static void run_steps(flp_propagator* h, uint64_t n) {
    ensure_conv_mode(h);
    while (n >= uint64_t(GRAPH_STEPS)) {
        if (!h->graph[h->cur]) build_graph(h);
        CK(cudaGraphLaunch(h->graph[h->cur], h->st));
        h->advance_clock(GRAPH_STEPS);
        n -= GRAPH_STEPS;
    }
    for (uint64_t i = 0; i < n; ++i) {
        if (!h->graph1[h->cur]) build_graph1(h);
        CK(cudaGraphLaunch(h->graph1[h->cur], h->st));
        h->cur ^= 1;
        h->advance_clock(1);
    }
}

static void invalidate_graphs(flp_propagator* h) {
    for (auto& g : h->graph)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    for (auto& g : h->graph1)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

static void prof_hook(flp_propagator* h, int stage) {
    CK(cudaEventRecord(h->prof_ev[h->prof_base + 1 + stage], h->st));
}

static void profile_run(flp_propagator* h, int steps, int flush, float* stage_ms, int max_stages, int* n_stages,
                        char* names, size_t names_len, float* step_ms) {
    std::vector<std::string> nm = h->stage_names();
    const int ns = int(nm.size());
    // Up to RING steps in flight, each with its own ns+1 events, so that the
    // host enqueues ahead and the device never waits for a launch inside a
    // timed step; the L2 flush of a step is enqueued between the previous
    // step's last event and this step's first one.
    constexpr int RING = 32;
    const int E = ns + 1;
    while (int(h->prof_ev.size()) < RING * E) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        h->prof_ev.push_back(e);
    }
    if (flush && !h->flush_buf) {
        int dev = 0, l2 = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
        h->flush_bytes = std::max<size_t>(size_t(2) * size_t(l2), size_t(64) << 20);
        CK(flp::dmalloc(&h->flush_buf, h->flush_bytes));
    }
    std::vector<double> acc(ns, 0.0);
    double total = 0.0;
    // Without stage_ms only the step is bracketed: no events between kernels.
    const bool staged = stage_ms != nullptr;
    auto harvest = [&](int slot) {
        cudaEvent_t* ev = h->prof_ev.data() + size_t(slot) * E;
        CK(cudaEventSynchronize(ev[ns]));
        for (int i = 0; staged && i < ns; ++i) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
            acc[i] += ms;
        }
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev[0], ev[ns]));
        total += ms;
    };
    h->hook = staged ? prof_hook : nullptr;
    try {
        for (int s = 0; s < steps; ++s) {
            const int slot = s % RING;
            if (s >= RING) harvest(slot);
            if (flush) CK(cudaMemsetAsync(h->flush_buf, s & 0xFF, h->flush_bytes, h->st));
            h->prof_base = slot * E;
            CK(cudaEventRecord(h->prof_ev[h->prof_base], h->st));
            h->enqueue_step();
            if (!staged) CK(cudaEventRecord(h->prof_ev[h->prof_base + ns], h->st));
            h->advance_clock(1);
        }
        for (int s = std::max(0, steps - RING); s < steps; ++s) harvest(s % RING);
    } catch (...) {
        h->hook = nullptr;
        throw;
    }
    h->hook = nullptr;
    if (n_stages) *n_stages = ns;
    for (int i = 0; i < ns && i < max_stages; ++i)
        if (stage_ms) stage_ms[i] = float(acc[i]);
    if (step_ms) *step_ms = float(total);
    if (names && names_len) {
        std::string joined;
        for (int i = 0; i < ns; ++i) joined += (i ? "," : "") + nm[i];
        std::strncpy(names, joined.c_str(), names_len - 1);
        names[names_len - 1] = 0;
    }
}

// Status words written by the kernels: reported once, then cleared.
static void check_status(flp_propagator* h) {
    int status = 0;
    CK(cudaMemcpy(&status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) {
        CK(cudaMemset(h->d_status, 0, sizeof(int)));
        if (status & STATUS_NONFINITE) throw FlpError(FLP_ERR_NONFINITE, "non-finite mass in the state");
    }
}

}  // namespace flp

// ------------------------------------------------------------------ C ABI ---
#define FLP_TRY(...)                                                      \
    try {                                                                 \
        __VA_ARGS__;                                                      \
        return FLP_OK;                                                    \
    } catch (const flp::FlpError& e) {                                    \
        flp::g_last_error = e.what();                                     \
        return e.code;                                                    \
    } catch (const flp::ConfigError& e) {                                 \
        flp::g_last_error = e.what();                                     \
        return FLP_ERR_INVALID_CONFIG;                                    \
    } catch (const std::bad_alloc&) {                                     \
        flp::g_last_error = "host allocation failed";                     \
        return FLP_ERR_OOM;                                               \
    } catch (const std::exception& e) {                                   \
        flp::g_last_error = e.what();                                     \
        return FLP_ERR_INVALID_ARGUMENT;                                  \
    }

#define FLP_CHECK_HANDLE(h)                                                    \
    if (!(h)) {                                                                \
        flp::g_last_error = "null handle";                                     \
        return FLP_ERR_INVALID_ARGUMENT;                                       \
    }

extern "C" {

const char* flp_last_error(void) { return flp::g_last_error.c_str(); }

int flp_create(const char* config_json, flp_propagator** out) {
    if (!config_json || !out) {
        flp::g_last_error = "null argument";
        return FLP_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    flp_propagator* h = new flp_propagator();
    try {
        flp::create(config_json, h);
    } catch (...) {
        h->free_all();
        delete h;
        FLP_TRY(throw)
    }
    *out = h;
    return FLP_OK;
}

int flp_destroy(flp_propagator* h) {
    if (!h) return FLP_OK;
    cudaStreamSynchronize(h->st);
    h->free_all();
    delete h;
    return FLP_OK;
}

int flp_seed_generate(const char* config_json, const char* seed_json, float* out, size_t n) {
    FLP_TRY({
        if (!config_json || !seed_json || !out) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "null argument");
        SimulationConfig c = parse_config(config_json);
        std::vector<float> g = generate_seed(seed_json, c);
        if (n != g.size()) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "output size mismatch: expected " + std::to_string(g.size()));
        std::memcpy(out, g.data(), g.size() * sizeof(float));
    })
}

int flp_state_from_seed(flp_propagator* h, const char* seed_json) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (!seed_json) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "null seed");
        std::vector<float> g = generate_seed(seed_json, h->cfg);
        upload_state(h, g.data(), g.size());
        h->time = 0.f;
        h->step = 0;
    })
}

int flp_write_state(flp_propagator* h, const float* state, size_t n, float time, uint64_t step) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (!state) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "null state");
        upload_state(h, state, n);
        h->time = time;
        h->step = step;
    })
}

int flp_read_state(flp_propagator* h, float* out, size_t n, float* time, uint64_t* step) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        const size_t CN = size_t(h->C) * h->N;
        if (!out || n != CN) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "state size mismatch: expected " + std::to_string(CN));
        CK(cudaMemcpyAsync(out, h->A[h->cur], CN * sizeof(float), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        if (time) *time = h->time;
        if (step) *step = h->step;
    })
}

int flp_step(flp_propagator* h) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY(run_steps(h, 1))
}

// The device address of a host buffer the device can read and write directly
// (page-locked memory under unified addressing), else nullptr.
static float* device_view_of_host(float* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // an unknown pointer is not an error of the handle
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost && a.devicePointer ? static_cast<float*>(a.devicePointer) : nullptr;
}

// step(&mut state) / run(&mut state, n) on a host state.  When the host buffer
// is device-addressable and the handle's path allows it (host_io_ok), the
// first step's row transforms read the source channels straight from it, so
// the transfer in overlaps their arithmetic (1.45e9 -> 1.47e9 cell-steps/s
// end to end at 512x512, C=3); otherwise the state is copied in.  The result
// is copied out: the gather writing it into the host buffer itself was
// measured slower than the copy (1.41e9).  Both ways give the same bits.
int flp_step_host(flp_propagator* h, float* state, size_t n, float* time, uint64_t* step, uint64_t steps) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        const size_t CN = size_t(h->C) * h->N;
        if (!state || n != CN) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "state size mismatch: expected " + std::to_string(CN));
        ensure_conv_mode(h);  // a pending measurement runs before the state is replaced
        float* hv = steps > 0 && h->host_io_ok() ? device_view_of_host(state) : nullptr;
        if (time) h->time = *time;
        if (step) h->step = *step;
        if (hv) {
            // channels that no kernel reads are not read by the row transforms
            for (int c = 0; c < h->C; ++c)
                if (std::find(h->h_srcs.begin(), h->h_srcs.end(), c) == h->h_srcs.end())
                    CK(cudaMemcpyAsync(h->A[h->cur] + size_t(c) * h->N, state + size_t(c) * h->N,
                                       h->N * sizeof(float), cudaMemcpyHostToDevice, h->st));
            h->enqueue_step(hv);
            h->advance_clock(1);
            run_steps(h, steps - 1);
        } else {
            CK(cudaMemcpyAsync(h->A[h->cur], state, CN * sizeof(float), cudaMemcpyHostToDevice, h->st));
            run_steps(h, steps);
        }
        CK(cudaMemcpyAsync(state, h->A[h->cur], CN * sizeof(float), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        if (time) *time = h->time;
        if (step) *step = h->step;
    })
}

int flp_run(flp_propagator* h, uint64_t n) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY(run_steps(h, n))
}

int flp_synchronize(flp_propagator* h) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        CK(cudaStreamSynchronize(h->st));
        check_status(h);
    })
}

int flp_synchronize_for(flp_propagator* h, double timeout_ms) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (!wait_stream_for(h->st, timeout_ms))
            throw FlpError(FLP_ERR_TIMEOUT, "the handle's stream did not finish within " +
                                                std::to_string(timeout_ms) + " ms");
        check_status(h);
    })
}

int flp_total_mass(flp_propagator* h, double* out) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (!out) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "null output");
        launch_mass_fp64(h->A[h->cur], size_t(h->C) * h->N, h->d_partial, h->np, h->d_mass, h->st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, h->d_mass, sizeof(double), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    })
}

int flp_total_mass_f32(flp_propagator* h, float* out) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (!out) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "null output");
        std::vector<float> s(size_t(h->C) * h->N);
        CK(cudaMemcpyAsync(s.data(), h->A[h->cur], s.size() * sizeof(float), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        float total = 0.f;
        for (int c = 0; c < h->C; ++c) {
            float m = 0.f;
            for (size_t i = 0; i < h->N; ++i) m += s[size_t(c) * h->N + i];
            total += m;
        }
        *out = total;
    })
}

int flp_get_info(flp_propagator* h, flp_info* out) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (!out) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "null output");
        out->width = h->W; out->height = h->H; out->depth = h->D;
        out->channels = h->C; out->n_kernels = h->K;
        ensure_conv_mode(h);
        out->conv_mode = h->conv_mode;
        out->time = h->time;
        out->step = h->step;
    })
}

int flp_get_tuning(flp_propagator* h, int32_t* out, int n) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (!out || n < FLP_TUNING_FIELDS) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "tuning needs 7 ints");
        ensure_conv_mode(h);
        const int32_t v[FLP_TUNING_FIELDS] = {h->conv_mode,         h->geom.wpc_r2c, h->geom.wpc_cols,
                                              h->geom.share_cols,   h->geom.wpc_c2r, h->gather_gby,
                                              h->tuning_cached ? 1 : 0};
        std::memcpy(out, v, sizeof(v));
    })
}

int flp_set_tuning(flp_propagator* h, const int32_t* in, int n) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (!in || n < FLP_TUNING_FIELDS - 1) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "tuning needs 6 ints");
        auto one_of = [](int v, int a, int b) { return v == a || v == b; };
        if (!one_of(in[0], FLP_CONV_DIRECT, FLP_CONV_FFT) || !one_of(in[1], 4, 8) || !one_of(in[2], 4, 8) ||
            !one_of(in[3], 0, 1) || !one_of(in[4], 4, 8) || !one_of(in[5], 1, 2))
            throw FlpError(FLP_ERR_INVALID_ARGUMENT, "tuning choice out of range");
        CK(cudaStreamSynchronize(h->st));
        ensure_conv_mode(h);
        if (h->K > 0) {
            if (in[0] == FLP_CONV_DIRECT && !h->direct_ok)
                throw FlpError(FLP_ERR_UNSUPPORTED, "direct convolution supports radius <= 24");
            if (in[0] == FLP_CONV_FFT && !h->fft_ok)
                throw FlpError(FLP_ERR_UNSUPPORTED, "FFT path needs an even width and sides of factors 2,3,5");
            h->conv_mode = in[0];
        }
        Tuning t;
        t.wpc_r2c = in[1];
        t.wpc_cols = in[2];
        t.share_cols = in[3];
        t.wpc_c2r = in[4];
        t.gather_gby = in[5];
        apply_tuning(h, t);
        h->tuning_cached = false;
        invalidate_graphs(h);
    })
}

int flp_set_conv_mode(flp_propagator* h, int mode) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (mode < FLP_CONV_AUTO || mode > FLP_CONV_FFT) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "bad conv mode");
        if (mode == FLP_CONV_AUTO) {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune_cache.erase({h->W, h->H, h->D, h->C, h->K, h->rmax, h->nsrc});
        }
        CK(cudaStreamSynchronize(h->st));
        resolve_conv_mode(h, mode);
        h->conv_pending = false;
        invalidate_graphs(h);
    })
}

void* flp_stream(flp_propagator* h) { return h ? static_cast<void*>(h->st) : nullptr; }

const float* flp_device_state(flp_propagator* h) { return h ? h->A[h->cur] : nullptr; }

int flp_device_info(char* pci_bus_id, int len, int* sm_count, size_t* l2_bytes) {
    FLP_TRY({
        int dev = 0;
        CK(cudaGetDevice(&dev));
        if (pci_bus_id && len > 0) CK(cudaDeviceGetPCIBusId(pci_bus_id, len, dev));
        if (sm_count) CK(cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, dev));
        if (l2_bytes) {
            int l2 = 0;
            CK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
            *l2_bytes = size_t(l2);
        }
    })
}

int flp_host_alloc(size_t bytes, void** out) {
    FLP_TRY({
        if (!out) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "null output");
        *out = nullptr;
        CK(cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault));
    })
}

int flp_host_free(void* p) {
    FLP_TRY({
        if (p) CK(cudaFreeHost(p));
    })
}

int flp_profile_run(flp_propagator* h, int steps, int flush_l2, float* stage_ms, int max_stages, int* n_stages,
                    char* names, size_t names_len, float* step_ms) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        if (steps < 0) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "negative step count");
        ensure_conv_mode(h);
        profile_run(h, steps, flush_l2, stage_ms, max_stages, n_stages, names, names_len, step_ms);
    })
}

int flp_debug_affinity(flp_propagator* h, float* aff_out, size_t n) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        const size_t CN = size_t(h->C) * h->N;
        if (!aff_out || n != CN) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "size mismatch");
        ensure_conv_mode(h);
        h->enqueue_conv(h->A[h->cur], nullptr);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(aff_out, h->U, CN * sizeof(float), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    })
}

int flp_debug_transport(flp_propagator* h, const float* state, const float* aff, float* out, size_t n) {
    FLP_CHECK_HANDLE(h);
    FLP_TRY({
        const size_t CN = size_t(h->C) * h->N;
        if (!state || !aff || !out || n != CN) throw FlpError(FLP_ERR_INVALID_ARGUMENT, "size mismatch");
        // The handle's own scratch planes are reused; the live state is untouched
        // (3D worlds go through the same entry: enqueue_transport dispatches).
        DevScratch scratch;
        float* a = scratch.add(dalloc<float>(CN));
        float* o = scratch.add(dalloc<float>(CN));
        CK(cudaMemcpyAsync(a, state, CN * sizeof(float), cudaMemcpyHostToDevice, h->st));
        CK(cudaMemcpyAsync(h->U, aff, CN * sizeof(float), cudaMemcpyHostToDevice, h->st));
        launch_zero_ints(h->d_dmax, 1, h->st);
        h->enqueue_transport(a, o);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, o, CN * sizeof(float), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    })
}

}  // extern "C"
