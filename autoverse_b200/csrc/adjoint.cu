// Differentiable step: forward T steps of a batch of same-shape 2D worlds with
// checkpoints, and the hand-written reverse sweep that returns dL/dA_0 and
// dL/d(parameters) for a loss gradient dL/dA_T given by the caller.
//
// Forward: the step kernels of the single-world engine, batched over worlds
// (plane p = world * C + channel; the FFT passes see B * nsrc sources and
// B * K kernels through their slot tables), so a world's trajectory is bit for
// bit the one CudaPropagator computes.  A_0, A_k, A_2k, ... are kept.
//
// Backward: segment by segment from the last checkpoint, the segment's states
// are recomputed, recording each step's convolution fields conv_k and the
// sources' column spectra, and then each step t is reversed:
//   1. U (growth of the recorded conv_k), the flow destinations and masses;
//   2. reintegration adjoint (per source) -> m^, F^;
//   3. flow adjoint -> gU^, gS^, S^_local, beta^;
//   4. Sobel transpose -> U^ and A^ = m^ + S^;
//   5. growth adjoint -> conv^, w^, mu^, sigma^;
//   6. convolution adjoint in the frequency domain: A^_src += IFFT(conj(K^)
//      FFT(conv^)); sum_t conj(A^_src) FFT(conv^) accumulates the kernel
//      correlation, inverted once at the end into K^ on the torus.
// Ring parameters (amplitude, distance, width) get their gradients on the
// host from K^ through the normalised ring-sum kernel (kernel.rs:32-92).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device_mem.h"
#include "adjoint.h"
#include "flowlenia_cuda.h"
#include "kernels.h"
#include "schema.h"

namespace flp {

extern thread_local std::string g_last_error;

namespace {

struct AdjError : std::runtime_error {
    int code;
    AdjError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw AdjError(e == cudaErrorMemoryAllocation ? FLP_ERR_OOM : FLP_ERR_CUDA,
                       std::string(what) + ": " + cudaGetErrorString(e));
}
#define CKA(x) ck((x), #x)

template <class T>
T* dalloc_a(size_t n) {
    void* p = nullptr;
    CKA(flp::dmalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    return static_cast<T*>(p);
}

void tw_push(std::vector<float2>& dst, int L, int count) {
    for (int t = 0; t < count; ++t) {
        const double ang = -2.0 * M_PI * double(t) / double(L);
        dst.push_back(make_float2(float(std::cos(ang)), float(std::sin(ang))));
    }
}

}  // namespace
}  // namespace flp

using namespace flp;

struct flp_adjoint {
    int B = 0, W = 0, H = 0, C = 0, K = 0, nsrc = 0, N = 0, P = 0;
    bool pow2 = true;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
    std::vector<SimulationConfig> cfgs;
    std::vector<std::vector<KernelStencil>> stencils;
    std::vector<int> src_of_slot;  // distinct source channels (same in every world)
    FftGeom g;
    float2* tw = nullptr;
    FlowParams* fps = nullptr;
    AdjKern* ak = nullptr;
    KDesc* kd = nullptr;
    int *srcs = nullptr, *slot = nullptr, *dmax = nullptr, *status = nullptr;
    float2 *KH = nullptr, *S = nullptr, *T = nullptr, *CBH = nullptr, *SB = nullptr, *KS = nullptr;
    float *U = nullptr, *DX = nullptr, *DY = nullptr, *conv = nullptr, *CB = nullptr;
    float *MBAR = nullptr, *FXB = nullptr, *FYB = nullptr, *GUX = nullptr, *GUY = nullptr, *UBAR = nullptr;
    float *GSX = nullptr, *GSY = nullptr, *SBL = nullptr;
    float* G[2] = {nullptr, nullptr};
    float* state0 = nullptr;
    float* fin = nullptr;
    float* work[2] = {nullptr, nullptr};
    std::vector<float*> ckpt, seg;
    // per step of the segment being reversed: the convolution fields conv_k
    // (B x K x N) and the column spectra of the sources (B x nsrc x spec),
    // recorded while the segment is recomputed from its checkpoint
    std::vector<float*> convseg;
    std::vector<float2*> ahseg;
    double* pg = nullptr;
    int steps = 0, every = 0;
    bool have_forward = false;
    float fwd_ms = 0.f, bwd_ms = 0.f;

    size_t CN() const { return size_t(B) * C * N; }
    size_t spec() const { return size_t(W / 2 + 1) * H; }

    void step(const float* a, float* an) {
        launch_fft_r2c(a, S, srcs, B * nsrc, W, H, g, dmax, B, st);
        launch_fft_cols_conv(S, KH, T, slot, B * nsrc, B * K, B, W, H, g, st);
        launch_fft_c2r_growth(T, U, kd, B * K, W, H, B * C, g, st);
        launch_flow_worlds(a, U, DX, DY, B, C, W, H, fps, dmax, status, st);
        launch_gather_worlds(DX, DY, a, an, B, C, W, H, fps, pow2, dmax, st);
    }

    // Step i of the segment being reversed, from a = A_t: records conv_k and
    // the sources' column spectra for its adjoint and, with an, advances to
    // A_t+1 (the same bits as step(): the growth of the recorded conv fields
    // is the fused growth's arithmetic).
    void record_step(const float* a, float* an, int i) {
        launch_fft_r2c(a, S, srcs, B * nsrc, W, H, g, dmax, B, st);
        launch_fft_cols(S, nullptr, ahseg[i], nullptr, B * nsrc, W, H, g, 1, 1.f, st);
        launch_fft_cols_conv(S, KH, T, slot, B * nsrc, B * K, B, W, H, g, st);
        launch_fft_c2r_raw(T, convseg[i], nullptr, B * K, W, H, 1.f, false, g, st);
        if (!an) return;
        launch_growth_worlds(convseg[i], U, ak, B, K, C, N, st);
        launch_flow_worlds(a, U, DX, DY, B, C, W, H, fps, dmax, status, st);
        launch_gather_worlds(DX, DY, a, an, B, C, W, H, fps, pow2, dmax, st);
    }

    // Reverse of step t (step i of its segment, recorded): a = A_t, gin =
    // dL/dA_{t+1} -> gout = dL/dA_t.
    void step_adjoint(const float* a, const float* gin, float* gout, int i) {
        const int nb = int(spec());
        const float* cv = convseg[i];
        // 1. U and the destinations from the recorded convolution fields
        launch_zero_ints(dmax, B, st);
        launch_growth_worlds(cv, U, ak, B, K, C, N, st);
        launch_flow_worlds(a, U, DX, DY, B, C, W, H, fps, dmax, status, st);
        // 2-4. transport adjoints
        launch_adj_reint(DX, DY, a, gin, MBAR, FXB, FYB, B, C, W, H, fps, pow2, st);
        launch_adj_flow(a, U, FXB, FYB, GUX, GUY, GSX, GSY, SBL, pg, P, B, C, W, H, fps, st);
        launch_adj_sobel_t(GUX, GUY, GSX, GSY, SBL, MBAR, UBAR, gout, B, C, W, H, st);
        // 5. growth adjoint
        launch_adj_growth(cv, UBAR, CB, ak, pg, P, B, K, C, N, st);
        // 6. convolution adjoint
        launch_fft_r2c(CB, T, nullptr, B * K, W, H, g, nullptr, 0, st);
        launch_fft_cols(T, nullptr, CBH, nullptr, B * K, W, H, g, 1, 1.f, st);
        launch_adj_spectral(KH, CBH, ahseg[i], SB, KS, ak, B, K, nsrc, nb, st);
        launch_fft_cols(SB, nullptr, SB, nullptr, B * nsrc, W, H, g, 2, 1.f, st);
        launch_fft_c2r_raw(SB, gout, srcs, B * nsrc, W, H, 1.f, true, g, st);
    }

    void free_all() {
        void* ptrs[] = {tw, fps, ak, kd, srcs, slot, dmax, status, KH, S, T, CBH, SB, KS, U, DX, DY, conv,
                        CB, MBAR, FXB, FYB, GUX, GUY, UBAR, GSX, GSY, SBL, G[0], G[1], state0, fin, work[0], work[1],
                        pg};
        for (void* p : ptrs)
            if (p) flp::dfree(p);
        for (float* p : ckpt) flp::dfree(p);
        for (float* p : seg) flp::dfree(p);
        for (float* p : convseg) flp::dfree(p);
        for (float2* p : ahseg) flp::dfree(p);
        ckpt.clear();
        seg.clear();
        convseg.clear();
        ahseg.clear();
        for (cudaEvent_t e : {e0, e1, e2, e3})
            if (e) cudaEventDestroy(e);
        if (st) cudaStreamDestroy(st);
    }
};

namespace flp {
namespace {

// Parameter-vector length of one world: beta_a, then per kernel weight, mu,
// sigma and per ring amplitude, distance, width.
int param_count(const SimulationConfig& c) {
    int n = 1;
    for (const auto& k : c.kernels) n += 3 + 3 * int(k.rings.size());
    return n;
}

void adj_create(flp_adjoint* h, const char* const* jsons, int n) {
    if (n < 1) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "need at least one world");
    for (int w = 0; w < n; ++w) {
        if (!jsons[w]) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "null config");
        h->cfgs.push_back(parse_config(jsons[w]));
    }
    const SimulationConfig& c0 = h->cfgs[0];
    if (c0.is_3d()) throw AdjError(FLP_ERR_UNSUPPORTED, "the differentiable step covers 2D worlds");
    h->B = n;
    h->W = c0.width;
    h->H = c0.height;
    h->C = c0.channels;
    h->K = int(c0.kernels.size());
    h->N = c0.width * c0.height;
    if (h->C > ADJ_MAX_CHANNELS) throw AdjError(FLP_ERR_UNSUPPORTED, "at most 8 channels per differentiable world");
    if (h->K == 0) throw AdjError(FLP_ERR_UNSUPPORTED, "a differentiable world needs at least one kernel");
    if (h->W % 2 || !fft_row_templated(h->W / 2) || !fft_col_templated(h->H))
        throw AdjError(FLP_ERR_UNSUPPORTED, "differentiable worlds need W/2 in {16..256} and H in {32..512}");
    for (const auto& c : h->cfgs) {
        if (c.width != h->W || c.height != h->H || c.depth != 1 || c.channels != h->C ||
            int(c.kernels.size()) != h->K || c.flow.distribution_size != c0.flow.distribution_size)
            throw AdjError(FLP_ERR_INVALID_CONFIG,
                           "worlds of one differentiable batch share width, height, channels, kernel count and "
                           "distribution_size");
        for (int k = 0; k < h->K; ++k)
            if (c.kernels[k].source_channel != c0.kernels[k].source_channel ||
                c.kernels[k].target_channel != c0.kernels[k].target_channel)
                throw AdjError(FLP_ERR_INVALID_CONFIG, "kernel source/target channels differ between worlds");
    }
    // distinct sources in first-use order; slot of each kernel
    std::vector<int> kslot(h->K);
    for (int k = 0; k < h->K; ++k) {
        const int s = c0.kernels[k].source_channel;
        auto it = std::find(h->src_of_slot.begin(), h->src_of_slot.end(), s);
        if (it == h->src_of_slot.end()) { kslot[k] = int(h->src_of_slot.size()); h->src_of_slot.push_back(s); }
        else kslot[k] = int(it - h->src_of_slot.begin());
    }
    h->nsrc = int(h->src_of_slot.size());
    h->P = 1 + 3 * h->K;
    CKA(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&h->e0, &h->e1, &h->e2, &h->e3}) CKA(cudaEventCreate(e));
    transport_2d_set_attributes();
    fft2d_set_attributes(200 * 1024);
    adjoint_set_attributes();
    // FFT geometry and twiddles
    const int M = h->W / 2, Wc = M + 1;
    make_plan(M, h->g.pm);
    make_plan(h->H, h->g.ph);
    std::vector<float2> tw;
    tw_push(tw, M, M);
    tw_push(tw, h->W, Wc);
    tw_push(tw, h->H, h->H);
    h->tw = dalloc_a<float2>(tw.size());
    CKA(cudaMemcpy(h->tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice));
    h->g.twM = h->tw;
    h->g.twW = h->tw + M;
    h->g.twH = h->tw + M + Wc;
    // 4-warp CTAs for the FFT passes of the whole batch (throughput-bound, as
    // in the batched engine); the column pass transforms each source once
    h->g.wpc_r2c = h->g.wpc_cols = h->g.wpc_c2r = 4;
    h->g.share_cols = 1;
    // per-world tables
    std::vector<FlowParams> fps;
    std::vector<AdjKern> ak;
    std::vector<KDesc> kd;
    std::vector<int> srcs, slots;
    for (int w = 0; w < n; ++w) {
        const SimulationConfig& c = h->cfgs[w];
        FlowParams fp = flow_params_of(c);
        if (w == 0) h->pow2 = fp.area_pow2 != 0;
        fps.push_back(fp);
        h->stencils.emplace_back();
        for (int k = 0; k < h->K; ++k) {
            const KernelConfig& kc = c.kernels[k];
            h->stencils[w].push_back(build_kernel(kc, c.kernel_radius, 2));
            (void)pad_kernel(h->stencils[w].back(), h->W, h->H, 1);  // radius check
            AdjKern a{};
            a.weight = kc.weight;
            a.mu = kc.mu;
            a.sigma = kc.sigma;
            a.inv2s2 = 1.0f / (2.0f * kc.sigma * kc.sigma);
            a.src = kc.source_channel;
            a.tgt = kc.target_channel;
            a.slot = kslot[k];
            ak.push_back(a);
            KDesc d{};
            d.src = w * h->C + kc.source_channel;
            d.tgt = w * h->C + kc.target_channel;
            d.r = h->stencils[w].back().radius;
            d.weight = kc.weight;
            d.mu = kc.mu;
            d.inv2s2 = a.inv2s2;
            kd.push_back(d);
            slots.push_back(w * h->nsrc + kslot[k]);
        }
        for (int s = 0; s < h->nsrc; ++s) srcs.push_back(w * h->C + h->src_of_slot[s]);
    }
    h->fps = dalloc_a<FlowParams>(n);
    h->ak = dalloc_a<AdjKern>(ak.size());
    h->kd = dalloc_a<KDesc>(kd.size());
    h->srcs = dalloc_a<int>(srcs.size());
    h->slot = dalloc_a<int>(slots.size());
    CKA(cudaMemcpy(h->fps, fps.data(), fps.size() * sizeof(FlowParams), cudaMemcpyHostToDevice));
    CKA(cudaMemcpy(h->ak, ak.data(), ak.size() * sizeof(AdjKern), cudaMemcpyHostToDevice));
    CKA(cudaMemcpy(h->kd, kd.data(), kd.size() * sizeof(KDesc), cudaMemcpyHostToDevice));
    CKA(cudaMemcpy(h->srcs, srcs.data(), srcs.size() * sizeof(int), cudaMemcpyHostToDevice));
    CKA(cudaMemcpy(h->slot, slots.data(), slots.size() * sizeof(int), cudaMemcpyHostToDevice));
    h->dmax = dalloc_a<int>(n);
    h->status = dalloc_a<int>(1);
    CKA(cudaMemset(h->status, 0, sizeof(int)));
    // buffers
    const size_t sp = h->spec(), CN = h->CN(), BN = size_t(n) * h->N, BK = size_t(n) * h->K;
    const size_t nsl = size_t(n) * h->nsrc;
    h->KH = dalloc_a<float2>(sp * BK);
    h->S = dalloc_a<float2>(sp * nsl);
    h->T = dalloc_a<float2>(sp * BK);
    h->CBH = dalloc_a<float2>(sp * BK);
    h->SB = dalloc_a<float2>(sp * nsl);
    h->KS = dalloc_a<float2>(sp * BK);
    for (float** p : {&h->U, &h->DX, &h->DY, &h->MBAR, &h->FXB, &h->FYB, &h->GUX, &h->GUY, &h->UBAR,
                      &h->G[0], &h->G[1], &h->state0, &h->fin, &h->work[0], &h->work[1]})
        *p = dalloc_a<float>(CN);
    h->conv = dalloc_a<float>(BK * h->N);
    h->CB = dalloc_a<float>(BK * h->N);
    for (float** p : {&h->GSX, &h->GSY, &h->SBL}) *p = dalloc_a<float>(BN);
    h->pg = dalloc_a<double>(size_t(n) * h->P);
    CKA(cudaMemset(h->state0, 0, CN * sizeof(float)));
    // kernel spectra, scaled by 1/(W*H) as in the single-world engine
    std::vector<float> padded(BK * h->N);
    for (int w = 0; w < n; ++w)
        for (int k = 0; k < h->K; ++k) {
            std::vector<float> pk = pad_kernel(h->stencils[w][k], h->W, h->H, 1);
            std::copy(pk.begin(), pk.end(), padded.begin() + (size_t(w) * h->K + k) * h->N);
        }
    CKA(cudaMemcpyAsync(h->conv, padded.data(), padded.size() * sizeof(float), cudaMemcpyHostToDevice, h->st));
    launch_fft_r2c(h->conv, h->T, nullptr, int(BK), h->W, h->H, h->g, nullptr, 0, h->st);
    launch_fft_cols(h->T, nullptr, h->KH, nullptr, int(BK), h->W, h->H, h->g, 1,
                    float(1.0 / (double(h->W) * double(h->H))), h->st);
    CKA(cudaGetLastError());
    CKA(cudaStreamSynchronize(h->st));
}

void check_world(flp_adjoint* h, int w, size_t n) {
    if (w < 0 || w >= h->B) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "world index out of range");
    if (n != size_t(h->C) * h->N) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "state size mismatch");
}

void adj_forward(flp_adjoint* h, int steps, int every) {
    if (steps < 1 || every < 1) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "steps and checkpoint interval must be >= 1");
    const size_t CN = h->CN();
    const int nck = (steps + every - 1) / every;
    while (int(h->ckpt.size()) < nck) h->ckpt.push_back(dalloc_a<float>(CN));
    while (int(h->seg.size()) < every) h->seg.push_back(dalloc_a<float>(CN));
    while (int(h->convseg.size()) < every) h->convseg.push_back(dalloc_a<float>(size_t(h->B) * h->K * h->N));
    while (int(h->ahseg.size()) < every) h->ahseg.push_back(dalloc_a<float2>(size_t(h->B) * h->nsrc * h->spec()));
    CKA(cudaEventRecord(h->e0, h->st));
    CKA(cudaMemcpyAsync(h->ckpt[0], h->state0, CN * sizeof(float), cudaMemcpyDeviceToDevice, h->st));
    const float* a = h->ckpt[0];
    for (int t = 0; t < steps; ++t) {
        float* an;
        if (t + 1 == steps) an = h->fin;
        else if ((t + 1) % every == 0) an = h->ckpt[(t + 1) / every];
        else an = h->work[t & 1];
        h->step(a, an);
        a = an;
    }
    CKA(cudaEventRecord(h->e1, h->st));
    CKA(cudaGetLastError());
    CKA(cudaEventSynchronize(h->e1));
    CKA(cudaEventElapsedTime(&h->fwd_ms, h->e0, h->e1));
    int status = 0;
    CKA(cudaMemcpy(&status, h->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status & STATUS_NONFINITE) throw AdjError(FLP_ERR_NONFINITE, "non-finite mass or flow in the forward pass");
    h->steps = steps;
    h->every = every;
    h->have_forward = true;
}

// Ring-parameter gradients of one kernel from dL/dK on the torus (double).
// K = raw / sum(raw), raw(d) = sum_r b_r exp(-(nd - a_r)^2 / (2 w_r^2)) for
// nd = |d| / radius <= 1 (kernel.rs:32-80).
void ring_grads(const KernelConfig& kc, const KernelStencil& ks, const float* kbar, int W, int H, double* out) {
    const int r = ks.radius, size = ks.size;
    const size_t nr = kc.rings.size();
    std::vector<double> raw(size_t(size) * size, 0.0), kb(size_t(size) * size, 0.0), nd(size_t(size) * size, 0.0);
    std::vector<char> inside(size_t(size) * size, 0);
    double Z = 0.0;
    for (int y = 0; y < size; ++y)
        for (int x = 0; x < size; ++x) {
            const size_t i = size_t(y) * size + x;
            const double dx = x - r, dy = y - r;
            const double d = std::sqrt(dx * dx + dy * dy) / (r > 0 ? r : 1);
            nd[i] = d;
            const int ty = ((y - r) % H + H) % H, tx = ((x - r) % W + W) % W;
            kb[i] = kbar[size_t(ty) * W + tx];
            if (d > 1.0) continue;
            inside[i] = 1;
            double v = 0.0;
            for (const auto& rg : kc.rings) {
                const double t = d - rg.distance;
                v += double(rg.amplitude) * std::exp(-t * t / (2.0 * double(rg.width) * rg.width));
            }
            raw[i] = v;
            Z += v;
        }
    for (size_t j = 0; j < 3 * nr; ++j) out[j] = 0.0;
    if (!(Z > 0.0)) return;
    double dot = 0.0;
    for (size_t i = 0; i < raw.size(); ++i) dot += kb[i] * raw[i] / Z;
    for (size_t i = 0; i < raw.size(); ++i) {
        if (!inside[i]) continue;
        const double rb = (kb[i] - dot) / Z;  // dL/draw
        for (size_t j = 0; j < nr; ++j) {
            const auto& rg = kc.rings[j];
            const double b = rg.amplitude, a = rg.distance, w = rg.width;
            const double t = nd[i] - a;
            const double e = std::exp(-t * t / (2.0 * w * w));
            out[3 * j + 0] += rb * e;
            out[3 * j + 1] += rb * b * e * t / (w * w);
            out[3 * j + 2] += rb * b * e * t * t / (w * w * w);
        }
    }
}

void adj_backward(flp_adjoint* h, const float* dl_dfinal, float* dl_dinit, double* dl_dparams) {
    if (!h->have_forward) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "backward needs a forward pass first");
    const size_t CN = h->CN(), sp = h->spec(), BK = size_t(h->B) * h->K;
    CKA(cudaEventRecord(h->e2, h->st));
    CKA(cudaMemcpyAsync(h->G[0], dl_dfinal, CN * sizeof(float), cudaMemcpyHostToDevice, h->st));
    CKA(cudaMemsetAsync(h->KS, 0, sp * BK * sizeof(float2), h->st));
    CKA(cudaMemsetAsync(h->pg, 0, size_t(h->B) * h->P * sizeof(double), h->st));
    int cur = 0;
    const int nck = (h->steps + h->every - 1) / h->every;
    for (int j = nck - 1; j >= 0; --j) {
        const int t0 = j * h->every, t1 = std::min(t0 + h->every, h->steps);
        // segment states: seg[i] = A_{t0+i} for 0 < i < t1 - t0 (A_{t0} is the
        // checkpoint), recomputed with every step's convolution recorded
        const float* base = h->ckpt[j];
        const int n = t1 - t0;
        for (int i = 0; i < n; ++i)
            h->record_step(i == 0 ? base : h->seg[i], i + 1 < n ? h->seg[i + 1] : nullptr, i);
        for (int t = t1 - 1; t >= t0; --t) {
            const float* a = t == t0 ? base : h->seg[t - t0];
            h->step_adjoint(a, h->G[cur], h->G[cur ^ 1], t - t0);
            cur ^= 1;
        }
    }
    // kernel gradients on the torus: IFFT(sum_t conj(A^) CB^) / (W*H)
    launch_fft_cols(h->KS, nullptr, h->KS, nullptr, int(BK), h->W, h->H, h->g, 2, 1.f, h->st);
    launch_fft_c2r_raw(h->KS, h->conv, nullptr, int(BK), h->W, h->H, float(1.0 / (double(h->W) * double(h->H))),
                       false, h->g, h->st);
    CKA(cudaEventRecord(h->e3, h->st));
    CKA(cudaGetLastError());
    if (dl_dinit)
        CKA(cudaMemcpyAsync(dl_dinit, h->G[cur], CN * sizeof(float), cudaMemcpyDeviceToHost, h->st));
    std::vector<double> pg(size_t(h->B) * h->P);
    std::vector<float> kbar(BK * h->N);
    CKA(cudaMemcpyAsync(pg.data(), h->pg, pg.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    if (dl_dparams)
        CKA(cudaMemcpyAsync(kbar.data(), h->conv, kbar.size() * sizeof(float), cudaMemcpyDeviceToHost, h->st));
    CKA(cudaStreamSynchronize(h->st));
    CKA(cudaEventElapsedTime(&h->bwd_ms, h->e2, h->e3));
    if (!dl_dparams) return;
    size_t o = 0;
    for (int w = 0; w < h->B; ++w) {
        const SimulationConfig& c = h->cfgs[w];
        const double* q = pg.data() + size_t(w) * h->P;
        dl_dparams[o++] = q[0];
        for (int k = 0; k < h->K; ++k) {
            dl_dparams[o++] = q[1 + 3 * k];
            dl_dparams[o++] = q[2 + 3 * k];
            dl_dparams[o++] = q[3 + 3 * k];
            ring_grads(c.kernels[k], h->stencils[w][k], kbar.data() + (size_t(w) * h->K + k) * h->N, h->W, h->H,
                       dl_dparams + o);
            o += 3 * c.kernels[k].rings.size();
        }
    }
}

int afail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace
}  // namespace flp

#define ADJ_TRY(...)                                                 \
    try {                                                            \
        __VA_ARGS__;                                                 \
        return FLP_OK;                                               \
    } catch (const AdjError& e) {                                    \
        return afail(e.code, e.what());                              \
    } catch (const flp::ConfigError& e) {                            \
        return afail(FLP_ERR_INVALID_CONFIG, e.what());              \
    } catch (const std::bad_alloc&) {                                \
        return afail(FLP_ERR_OOM, "host allocation failed");         \
    } catch (const std::exception& e) {                              \
        return afail(FLP_ERR_INVALID_ARGUMENT, e.what());            \
    }

#define ADJ_HANDLE(h) \
    if (!(h)) return afail(FLP_ERR_INVALID_ARGUMENT, "null adjoint handle");

extern "C" {

int flp_adj_create(const char* const* config_jsons, int n_worlds, flp_adjoint** out) {
    if (!config_jsons || !out) return afail(FLP_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    flp_adjoint* h = new flp_adjoint();
    try {
        adj_create(h, config_jsons, n_worlds);
    } catch (...) {
        h->free_all();
        delete h;
        ADJ_TRY(throw)
    }
    *out = h;
    return FLP_OK;
}

int flp_adj_destroy(flp_adjoint* h) {
    if (!h) return FLP_OK;
    cudaStreamSynchronize(h->st);
    h->free_all();
    delete h;
    return FLP_OK;
}

int flp_adj_write_state(flp_adjoint* h, int world, const float* state, size_t n) {
    ADJ_HANDLE(h);
    ADJ_TRY({
        check_world(h, world, n);
        if (!state) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "null state");
        CKA(cudaMemcpyAsync(h->state0 + size_t(world) * h->C * h->N, state, n * sizeof(float),
                            cudaMemcpyHostToDevice, h->st));
        CKA(cudaStreamSynchronize(h->st));
        h->have_forward = false;
    })
}

int flp_adj_state_from_seed(flp_adjoint* h, int world, const char* seed_json) {
    ADJ_HANDLE(h);
    ADJ_TRY({
        if (world < 0 || world >= h->B || !seed_json) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "bad argument");
        std::vector<float> s = generate_seed(seed_json, h->cfgs[world]);
        CKA(cudaMemcpyAsync(h->state0 + size_t(world) * h->C * h->N, s.data(), s.size() * sizeof(float),
                            cudaMemcpyHostToDevice, h->st));
        CKA(cudaStreamSynchronize(h->st));
        h->have_forward = false;
    })
}

int flp_adj_forward(flp_adjoint* h, int steps, int checkpoint_every) {
    ADJ_HANDLE(h);
    ADJ_TRY(adj_forward(h, steps, checkpoint_every))
}

int flp_adj_read_final(flp_adjoint* h, int world, float* out, size_t n) {
    ADJ_HANDLE(h);
    ADJ_TRY({
        check_world(h, world, n);
        if (!out) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "null output");
        if (!h->have_forward) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "no forward pass yet");
        CKA(cudaMemcpyAsync(out, h->fin + size_t(world) * h->C * h->N, n * sizeof(float), cudaMemcpyDeviceToHost,
                            h->st));
        CKA(cudaStreamSynchronize(h->st));
    })
}

int flp_adj_param_count(flp_adjoint* h, int world, int* count) {
    ADJ_HANDLE(h);
    ADJ_TRY({
        if (world < 0 || world >= h->B || !count) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "bad argument");
        *count = param_count(h->cfgs[world]);
    })
}

int flp_adj_backward(flp_adjoint* h, const float* dl_dfinal, size_t n, float* dl_dinitial, size_t n_initial,
                     double* dl_dparams, size_t n_params) {
    ADJ_HANDLE(h);
    ADJ_TRY({
        if (!dl_dfinal || n != h->CN()) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "dL/dA_T size mismatch");
        if (dl_dinitial && n_initial != h->CN()) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "dL/dA_0 size mismatch");
        size_t np = 0;
        for (const auto& c : h->cfgs) np += size_t(param_count(c));
        if (dl_dparams && n_params != np) throw AdjError(FLP_ERR_INVALID_ARGUMENT, "parameter gradient size mismatch");
        adj_backward(h, dl_dfinal, dl_dinitial, dl_dparams);
    })
}

int flp_adj_timings(flp_adjoint* h, float* forward_ms, float* backward_ms) {
    ADJ_HANDLE(h);
    if (forward_ms) *forward_ms = h->fwd_ms;
    if (backward_ms) *backward_ms = h->bwd_ms;
    return FLP_OK;
}

}  // extern "C"
