// Animation recorder: the reference's AnimationRecorder (src/animation/
// recorder.rs:56-200) writing its FLWA files (src/animation/format.rs) from a
// single-world handle's device state, without stalling the step stream.
//
// record() enqueues, on the handle's stream right after the steps enqueued so
// far, a device-to-device copy of the state into a slot of a device ring; a
// copy stream waits for it and moves the slot into pinned host memory; a
// writer thread waits for that copy and appends the frame to the file.  The
// handle's stream only ever waits for the fast device copy, so steps keep
// running while frames cross PCIe and reach the disk; record() blocks only
// when every slot is still in flight.  Frames are the state's channels, f32
// little-endian (the device's own byte order), exactly as encode_frame
// (format.rs:171-178) lays them out; frame offsets are known when a frame is
// enqueued, and finalize() appends the index table and rewrites the header
// with the frame count, as the reference does.
#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "device_mem.h"
#include "flowlenia_cuda.h"
#include "kernels.h"

namespace flp {

extern thread_local std::string g_last_error;

namespace {

constexpr uint32_t FLWA_VERSION = 1;   // format.rs:9
constexpr size_t FLWA_HEADER = 52;     // format.rs:78-81
constexpr int REC_SLOTS = 4;           // frames in flight

void ckr(cudaError_t e, const char* what) { throw_cuda(e, what); }

struct UnsupportedRec : std::runtime_error {
    using std::runtime_error::runtime_error;
};

template <class T>
void put(unsigned char*& p, T v) {  // little-endian on every platform this library builds for
    std::memcpy(p, &v, sizeof v);
    p += sizeof v;
}

// AnimationHeader::write_to (format.rs:95-108)
void header_bytes(unsigned char out[FLWA_HEADER], uint32_t w, uint32_t h, uint32_t d, uint32_t c, uint64_t frames,
                  float dt) {
    unsigned char* p = out;
    std::memcpy(p, "FLWA", 4);
    p += 4;
    put<uint16_t>(p, FLWA_VERSION);
    put<uint16_t>(p, 0);  // flags: no compression, no delta encoding (recorder.rs:84-87)
    put<uint32_t>(p, w);
    put<uint32_t>(p, h);
    put<uint32_t>(p, d);
    put<uint32_t>(p, c);
    put<uint64_t>(p, frames);
    put<float>(p, dt);
    std::memset(p, 0, 16);  // reserved
}

}  // namespace
}  // namespace flp

using namespace flp;

struct flp_recorder {
    flp_propagator* h = nullptr;
    FILE* f = nullptr;
    uint32_t W = 0, H = 0, D = 1, C = 0;
    float dt = 0.f;
    size_t frame_bytes = 0;
    uint32_t frame_skip = 1;
    uint64_t max_frames = 0;
    uint32_t step_counter = 0;
    uint64_t frames_written = 0;  // frames enqueued
    int device = 0;
    cudaStream_t copy = nullptr;
    float* dslot[REC_SLOTS] = {nullptr};
    float* hslot[REC_SLOTS] = {nullptr};
    cudaEvent_t ev_snap[REC_SLOTS] = {nullptr};
    cudaEvent_t ev_host[REC_SLOTS] = {nullptr};
    bool busy[REC_SLOTS] = {false};
    // writer thread
    std::thread writer;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<int> queue;  // slots to write, in frame order
    bool stop = false;
    std::string io_error;

    void writer_loop() {
        cudaSetDevice(device);
        for (;;) {
            int slot;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (queue.empty()) return;
                slot = queue.front();
            }
            const cudaError_t e = cudaEventSynchronize(ev_host[slot]);
            bool ok = e == cudaSuccess && io_error.empty();
            if (ok) ok = std::fwrite(hslot[slot], 1, frame_bytes, f) == frame_bytes;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (!ok && io_error.empty())
                    io_error = e != cudaSuccess ? std::string("frame copy: ") + cudaGetErrorString(e) : "frame write failed";
                queue.pop_front();
                busy[slot] = false;
            }
            cv.notify_all();
        }
    }

    // record_frame (recorder.rs:109-166): returns whether a frame was taken
    bool record() {
        ++step_counter;
        if (step_counter < frame_skip) return false;
        step_counter = 0;
        if (max_frames > 0 && frames_written >= max_frames) return false;
        const int slot = int(frames_written % REC_SLOTS);
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return !busy[slot]; });
            if (!io_error.empty()) throw std::runtime_error(io_error);
            busy[slot] = true;
        }
        const PropView v = prop_view(h);
        ckr(cudaMemcpyAsync(dslot[slot], v.state, frame_bytes, cudaMemcpyDeviceToDevice, v.stream), "frame snapshot");
        ckr(cudaEventRecord(ev_snap[slot], v.stream), "event");
        ckr(cudaStreamWaitEvent(copy, ev_snap[slot], 0), "event wait");
        ckr(cudaMemcpyAsync(hslot[slot], dslot[slot], frame_bytes, cudaMemcpyDeviceToHost, copy), "frame copy");
        ckr(cudaEventRecord(ev_host[slot], copy), "event");
        {
            std::lock_guard<std::mutex> lk(mu);
            queue.push_back(slot);
        }
        cv.notify_all();
        ++frames_written;
        return true;
    }

    void drain() {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return queue.empty(); });
    }

    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        if (writer.joinable()) writer.join();
    }

    void free_all() {
        shutdown();
        if (copy) cudaStreamSynchronize(copy);
        for (int i = 0; i < REC_SLOTS; ++i) {
            if (dslot[i]) flp::dfree(dslot[i]);
            if (hslot[i]) cudaFreeHost(hslot[i]);
            if (ev_snap[i]) cudaEventDestroy(ev_snap[i]);
            if (ev_host[i]) cudaEventDestroy(ev_host[i]);
        }
        if (copy) cudaStreamDestroy(copy);
        if (f) std::fclose(f);
        f = nullptr;
    }
};

namespace flp {
namespace {

void rec_create(flp_recorder* r, flp_propagator* h, const char* path, int compression, uint32_t frame_skip,
                uint64_t max_frames) {
    if (compression == 1)  // the reference without its optional lz4 feature (recorder.rs:62-69)
        throw UnsupportedRec("LZ4 compression requested but 'lz4' feature is not enabled");
    if (compression != 0) throw std::invalid_argument("unknown compression type");
    const PropView v = prop_view(h);
    r->h = h;
    r->W = uint32_t(v.width);
    r->H = uint32_t(v.height);
    r->D = uint32_t(v.depth);
    r->C = uint32_t(v.channels);
    r->dt = v.dt;
    r->device = v.device;
    r->frame_bytes = size_t(r->W) * r->H * r->D * r->C * sizeof(float);
    r->frame_skip = frame_skip;
    r->max_frames = max_frames;
    r->f = std::fopen(path, "wb");
    if (!r->f) throw std::invalid_argument(std::string("cannot create ") + path);
    unsigned char hdr[FLWA_HEADER];
    header_bytes(hdr, r->W, r->H, r->D, r->C, 0, r->dt);  // placeholder: frame count 0
    if (std::fwrite(hdr, 1, FLWA_HEADER, r->f) != FLWA_HEADER) throw std::runtime_error("header write failed");
    ckr(cudaStreamCreateWithFlags(&r->copy, cudaStreamNonBlocking), "stream");
    for (int i = 0; i < REC_SLOTS; ++i) {
        ckr(flp::dmalloc(&r->dslot[i], r->frame_bytes), "frame slot");
        ckr(cudaMallocHost(&r->hslot[i], r->frame_bytes), "pinned frame slot");
        ckr(cudaEventCreateWithFlags(&r->ev_snap[i], cudaEventDisableTiming), "event");
        ckr(cudaEventCreateWithFlags(&r->ev_host[i], cudaEventDisableTiming), "event");
    }
    r->writer = std::thread([r] { r->writer_loop(); });
}

// finalize (recorder.rs:171-200)
void rec_finalize(flp_recorder* r, uint64_t* frame_count, uint64_t* total_bytes, uint64_t* avg_frame) {
    r->drain();
    if (!r->io_error.empty()) throw std::runtime_error(r->io_error);
    const uint64_t n = r->frames_written;
    const uint64_t index_offset = FLWA_HEADER + n * uint64_t(r->frame_bytes);
    std::vector<unsigned char> idx(size_t(n) * 16);
    unsigned char* p = idx.data();
    for (uint64_t i = 0; i < n; ++i) {
        put<uint64_t>(p, FLWA_HEADER + i * uint64_t(r->frame_bytes));  // FrameIndex::write_to (format.rs:149-153)
        put<uint64_t>(p, uint64_t(r->frame_bytes));
    }
    if (n && std::fwrite(idx.data(), 1, idx.size(), r->f) != idx.size()) throw std::runtime_error("index write failed");
    unsigned char hdr[FLWA_HEADER];
    header_bytes(hdr, r->W, r->H, r->D, r->C, n, r->dt);
    if (std::fseek(r->f, 0, SEEK_SET) != 0 || std::fwrite(hdr, 1, FLWA_HEADER, r->f) != FLWA_HEADER ||
        std::fflush(r->f) != 0)
        throw std::runtime_error("header rewrite failed");
    if (frame_count) *frame_count = n;
    if (total_bytes) *total_bytes = index_offset + n * 16;
    if (avg_frame) *avg_frame = n ? (index_offset - FLWA_HEADER) / n : 0;
}

int rfail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace
}  // namespace flp

#define REC_TRY(...)                                             \
    try {                                                        \
        __VA_ARGS__;                                             \
        return FLP_OK;                                           \
    } catch (const flp::UnsupportedRec& e) {                     \
        return flp::rfail(FLP_ERR_UNSUPPORTED, e.what());        \
    } catch (const std::invalid_argument& e) {                   \
        return flp::rfail(FLP_ERR_INVALID_ARGUMENT, e.what());   \
    } catch (const flp::DeviceOom& e) {                          \
        return flp::rfail(FLP_ERR_OOM, e.what());                \
    } catch (const std::exception& e) {                          \
        return flp::rfail(FLP_ERR_CUDA, e.what());               \
    }

extern "C" {

int flp_rec_create(flp_propagator* h, const char* path, int compression, uint32_t frame_skip, uint64_t max_frames,
                   flp_recorder** out) {
    if (!h || !path || !out) return rfail(FLP_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    flp_recorder* r = new flp_recorder();
    try {
        rec_create(r, h, path, compression, frame_skip, max_frames);
    } catch (...) {
        r->free_all();
        delete r;
        REC_TRY(throw)
    }
    *out = r;
    return FLP_OK;
}

int flp_rec_record(flp_recorder* r, int* recorded) {
    if (!r) return rfail(FLP_ERR_INVALID_ARGUMENT, "null recorder");
    REC_TRY({
        const bool took = r->record();
        if (recorded) *recorded = took ? 1 : 0;
    })
}

int flp_rec_run(flp_recorder* r, uint64_t steps) {
    if (!r) return rfail(FLP_ERR_INVALID_ARGUMENT, "null recorder");
    for (uint64_t i = 0; i < steps; ++i) {
        const int rc = flp_run(r->h, 1);
        if (rc != FLP_OK) return rc;
        try {
            r->record();
        } catch (const std::exception& e) {
            return rfail(FLP_ERR_CUDA, e.what());
        }
    }
    return FLP_OK;
}

int flp_rec_frames_written(flp_recorder* r, uint64_t* n) {
    if (!r || !n) return rfail(FLP_ERR_INVALID_ARGUMENT, "null argument");
    *n = r->frames_written;
    return FLP_OK;
}

int flp_rec_finalize(flp_recorder* r, uint64_t* frame_count, uint64_t* total_bytes, uint64_t* avg_frame_bytes) {
    if (!r) return rfail(FLP_ERR_INVALID_ARGUMENT, "null recorder");
    int rc = FLP_OK;
    try {
        rec_finalize(r, frame_count, total_bytes, avg_frame_bytes);
    } catch (const std::exception& e) {
        rc = rfail(FLP_ERR_CUDA, e.what());
    }
    r->free_all();
    delete r;
    return rc;
}

}  // extern "C"
