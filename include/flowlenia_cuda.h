/*
 * flowlenia_cuda.h — C ABI of the B200 Flow Lenia step engine.
 *
 * Plain pointers and sizes only.  Every entry point returns an int status
 * (FLP_OK == 0, negative on failure) and never aborts the process; the text of
 * the last failure on the calling thread is available from flp_last_error().
 *
 * Each entry point names the reference interface it replaces (paths are
 * within the nathan-gage/autoverse crate).  Configs and seeds are the
 * reference's unchanged JSON schema (src/schema/config.rs:14-111,
 * src/schema/seed.rs:13-135).
 *
 * State layout on both sides of the boundary is the reference's
 * SimulationState layout: channel-major planes, each plane z*H*W + y*W + x
 * (src/compute/propagator.rs:18-21), f32.
 *
 * Threading: one handle per host thread.  All device work of a handle runs on
 * one CUDA stream owned by the handle; calls on different handles may run
 * concurrently.
 */
#ifndef FLOWLENIA_CUDA_H
#define FLOWLENIA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FLP_API __attribute__((visibility("default")))
#else
#define FLP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define FLP_OK 0
#define FLP_ERR_INVALID_CONFIG -1 /* config.rs:136-164 ConfigError, or bad JSON */
#define FLP_ERR_INVALID_ARGUMENT -2
#define FLP_ERR_OOM -3
#define FLP_ERR_CUDA -4
#define FLP_ERR_TIMEOUT -5   /* a bounded host wait (flp_*synchronize_for) ran out */
#define FLP_ERR_NONFINITE -6 /* NaN/Inf found in the state */
#define FLP_ERR_UNSUPPORTED -7

/* Convolution strategy (the reference always uses FFT, src/compute/fft.rs). */
#define FLP_CONV_AUTO 0   /* measured choice, cached per (grid, radius, channels) */
#define FLP_CONV_DIRECT 1 /* shared-memory tiled torus convolution */
#define FLP_CONV_FFT 2    /* batched real-to-complex Stockham FFT */

typedef struct flp_propagator flp_propagator;

typedef struct {
    int32_t width, height, depth, channels, n_kernels;
    int32_t conv_mode;      /* FLP_CONV_DIRECT or FLP_CONV_FFT once resolved */
    float time;             /* SimulationState.time, propagator.rs:28-29 */
    uint64_t step;          /* SimulationState.step, propagator.rs:30-31 */
} flp_info;

/* Text of the last error raised on this thread ("" if none). */
FLP_API const char* flp_last_error(void);

/* CudaPropagator::new — replaces CpuPropagator::new (src/compute/propagator.rs:157-236)
 * and CpuPropagator3D::new (src/compute/propagator3d.rs:49-116).  Validates like
 * SimulationConfig::validate (src/schema/config.rs:136-164) and returns
 * FLP_ERR_INVALID_CONFIG instead of panicking.  The state starts all zero. */
FLP_API int flp_create(const char* config_json, flp_propagator** out);

/* Drop. */
FLP_API int flp_destroy(flp_propagator* h);

/* SimulationState::from_seed (src/compute/propagator.rs:36-59, seed generation
 * src/schema/seed.rs:160-304): generate on the host and upload; time=0, step=0. */
FLP_API int flp_state_from_seed(flp_propagator* h, const char* seed_json);

/* Seed::generate without a propagator: fills out[channels*depth*height*width]. */
FLP_API int flp_seed_generate(const char* config_json, const char* seed_json, float* out, size_t n);

/* Replace the device state with a caller-owned host buffer (copied in). */
FLP_API int flp_write_state(flp_propagator* h, const float* state, size_t n, float time, uint64_t step);

/* Copy the device state out to a caller-owned host buffer; time/step may be NULL. */
FLP_API int flp_read_state(flp_propagator* h, float* out, size_t n, float* time, uint64_t* step);

/* CpuPropagator::step (src/compute/propagator.rs:239-420) and
 * CpuPropagator3D::step (src/compute/propagator3d.rs:119-308).  Asynchronous:
 * enqueues on the handle's stream. */
FLP_API int flp_step(flp_propagator* h);

/* CpuPropagator::run (src/compute/propagator.rs:423-427): n steps, replayed
 * from a captured CUDA graph.  Asynchronous. */
FLP_API int flp_run(flp_propagator* h, uint64_t n);

/* CpuPropagator::step / run on a state held in host memory, the form the
 * reference's callers use (step(&mut state), src/compute/propagator.rs:239):
 * copies state[channels*depth*height*width] in (with *time and *step when
 * given), advances `steps` steps, and copies the state and the advanced clock
 * back into the same buffers; one stream synchronisation.  With `state` in
 * pinned memory (flp_host_alloc or any device-addressable page-locked buffer)
 * the copy back is a DMA transfer and, on the 2D FFT path, the first step's
 * row transforms read the source channels straight from the buffer instead of
 * a copy in; the results are the same bits either way. */
FLP_API int flp_step_host(flp_propagator* h, float* state, size_t n, float* time, uint64_t* step, uint64_t steps);

/* Wait for the handle's stream; reports device-side status words
 * (FLP_ERR_NONFINITE when the bound check saw a non-finite mass). */
FLP_API int flp_synchronize(flp_propagator* h);

/* flp_synchronize with a limit: waits at most timeout_ms for the handle's
 * stream (host-side polling, no device spin) and returns FLP_ERR_TIMEOUT when
 * work is still pending; nothing is cancelled, so a later synchronize can
 * still wait for it.  A caller's watchdog for a stalled or overloaded device.
 * No counterpart in the reference (its step is synchronous). */
FLP_API int flp_synchronize_for(flp_propagator* h, double timeout_ms);

/* SimulationState::total_mass (src/compute/propagator.rs:80-82) computed on
 * the device as an FP64 compensated (Neumaier) sum over all channels. */
FLP_API int flp_total_mass(flp_propagator* h, double* out);

/* The reference's own f32 total_mass: sequential f32 sums per channel, then
 * summed over channels (src/compute/reintegration.rs:221-228). */
FLP_API int flp_total_mass_f32(flp_propagator* h, float* out);

FLP_API int flp_get_info(flp_propagator* h, flp_info* out);

/* Force a convolution strategy (FLP_CONV_*); FLP_CONV_AUTO re-runs the tuner. */
FLP_API int flp_set_conv_mode(flp_propagator* h, int mode);

/* Measured launch choices (the autotuner; none of them changes a result bit):
 *   0 convolution path (FLP_CONV_DIRECT / FLP_CONV_FFT)
 *   1 warps per CTA of the FFT row R2C pass (4 or 8)
 *   2 warps per CTA of the FFT column pass (4 or 8)
 *   3 column pass: 1 = one forward transform per source channel shared by
 *     the kernels that read it, 0 = one per kernel (more CTAs)
 *   4 warps per CTA of the FFT row C2R + growth pass (4 or 8)
 *   5 destination rows per thread of the 2D gather (1 or 2)
 *   6 (get only) 1 when the choices came from the process-wide cache of an
 *     earlier handle with the same shape (grid, channels, kernels, radius,
 *     source channels), 0 when this handle measured them.
 * The tuner runs on a handle's first step (or flp_set_conv_mode); the choices
 * are cached per shape for the process.  flp_set_tuning forces fields 0-5. */
#define FLP_TUNING_FIELDS 7
FLP_API int flp_get_tuning(flp_propagator* h, int32_t* out, int n);
FLP_API int flp_set_tuning(flp_propagator* h, const int32_t* in, int n);

/* The handle's cudaStream_t, for callers that time or order work around it. */
FLP_API void* flp_stream(flp_propagator* h);

/* Device pointer of the current state (channels*N floats) for zero-copy
 * callers; valid until the next step/run/write. */
FLP_API const float* flp_device_state(flp_propagator* h);

/* Current device's PCI bus id (for matching nvidia-smi samples), SM count and
 * L2 size. */
FLP_API int flp_device_info(char* pci_bus_id, int len, int* sm_count, size_t* l2_bytes);

/* Pinned (page-locked) host buffers for callers that stream states to and
 * from the device every step; flp_write_state/flp_read_state copy from and to
 * them at full PCIe/C2C bandwidth. */
FLP_API int flp_host_alloc(size_t bytes, void** out);
FLP_API int flp_host_free(void* p);

/* Measurement entry point: runs `steps` steps eagerly, each optionally
 * preceded by a write of a buffer twice the size of L2 (so every step starts
 * with a cold cache), with CUDA events on the handle's stream around every
 * kernel.  Writes the summed device time of each stage (ms) to stage_ms[i]
 * (up to max_stages entries), the stage names (comma-separated) to names,
 * the number of stages to n_stages and the summed step time to step_ms.
 * With stage_ms NULL only each step is bracketed (no events between its
 * kernels) and only step_ms (and n_stages, names) are written.
 * Synchronous. */
FLP_API int flp_profile_run(flp_propagator* h, int steps, int flush_l2, float* stage_ms, int max_stages,
                            int* n_stages, char* names, size_t names_len, float* step_ms);

/* Stage entry points used by stage-level parity tests.
 * Affinity U = sum_k w_k G(K_k * A_src) (src/compute/propagator.rs:244-279):
 * reads the current state, writes channels*N floats to the host buffer. */
FLP_API int flp_debug_affinity(flp_propagator* h, float* aff_out, size_t n);

/* Transport stage (propagator.rs:304-419) from a host state and host affinity:
 * mass sum, Sobel, flow, reintegration.  Writes the next state to out. */
FLP_API int flp_debug_transport(flp_propagator* h, const float* state, const float* aff, float* out, size_t n);

/* FP64 twin of one 2D step (CpuPropagator::step, propagator.rs:239-420, in
 * double): the engine's own direct convolution + growth, flow and gather
 * functions instantiated in double, with the config's f32 parameters widened.
 * No counterpart in the reference: it states the f32 engine's error against
 * an FP64 build of the same arithmetic.  Host buffers of channels*N doubles:
 * state in, next state out, affinity out (may be NULL).  Allocates and frees
 * its own device buffers; synchronous; diagnostic, not a product path. */
FLP_API int flp_twin64_step(const char* config_json, const double* state, double* affinity, double* next);

/* ---- Batched worlds ----------------------------------------------------
 * Many independent 2D worlds of uneven sizes, channel counts and parameters,
 * advanced together by persistent kernels that pull (world, tile) items from
 * device work queues; replaces running one CpuPropagator per candidate as the
 * reference's evolution search does (src/compute/evolution/search.rs:152-172,
 * src/compute/evolution/fitness.rs:26-88).  Each world follows
 * CpuPropagator::step (src/compute/propagator.rs:239-420) and gives the same
 * bits as a single-world flp_propagator with the same config.  Widths must
 * be even with W/2 in {16,24,32,48,64,96,128,192,256} and heights in
 * {32,48,64,96,128,192,256,384,512}. */
typedef struct flp_batch flp_batch;

FLP_API int flp_batch_create(const char* const* config_jsons, int n_worlds, flp_batch** out);
FLP_API int flp_batch_destroy(flp_batch* b);
/* New configs for an existing batch's worlds (the next generation of an
 * evolution run, evolution/search.rs:152-172, which builds one CpuPropagator
 * per candidate each generation): n_worlds must be the batch's count and every
 * world must keep its width, height, channel count and kernels' (source,
 * target) channel pairs, else FLP_ERR_INVALID_ARGUMENT and nothing changes;
 * an invalid config gives FLP_ERR_INVALID_CONFIG, also with nothing changed.
 * Growth and ring parameters, kernel radius, flow parameters and dt may all
 * change.  States are zeroed and time/step reset; the device pools, work
 * queues and captured graphs are reused. */
FLP_API int flp_batch_reconfigure(flp_batch* b, const char* const* config_jsons, int n_worlds);
/* SimulationState::from_seed for one world (time and step reset to 0). */
FLP_API int flp_batch_state_from_seed(flp_batch* b, int world, const char* seed_json);
/* The same for every world at once: seed_jsons[w] (NULL leaves world w as it
 * is), n = number of worlds; one host-to-device copy per run of seeded worlds. */
FLP_API int flp_batch_states_from_seeds(flp_batch* b, const char* const* seed_jsons, int n);
FLP_API int flp_batch_write_world(flp_batch* b, int world, const float* state, size_t n);
FLP_API int flp_batch_read_world(flp_batch* b, int world, float* out, size_t n, float* time, uint64_t* step);
/* CpuPropagator::run for every world at once; replays a captured CUDA graph. */
FLP_API int flp_batch_run(flp_batch* b, uint64_t n);
FLP_API int flp_batch_synchronize(flp_batch* b);
/* flp_batch_synchronize with a limit, as flp_synchronize_for. */
FLP_API int flp_batch_synchronize_for(flp_batch* b, double timeout_ms);
/* FP64 compensated total mass of every world (n = number of worlds). */
FLP_API int flp_batch_total_mass(flp_batch* b, double* per_world, int n);
FLP_API int flp_batch_info(flp_batch* b, int* n_worlds, size_t* cell_channels, size_t* cells);
/* Kernel spectra in the pool: worlds with the same grid and the same kernel
 * stencils (parameter sweeps over growth, flow or dt) share one set, computed
 * once.  Reports the number of distinct sets and their device bytes. */
FLP_API int flp_batch_kernel_spectra(flp_batch* b, int* unique_sets, size_t* bytes);
FLP_API void* flp_batch_stream(flp_batch* b);
/* Trajectory statistics for fitness evaluation (the quantities the reference's
 * FitnessEvaluator samples, src/compute/evolution/fitness.rs:96-240 and
 * 420-520), for every world at once, of the channel sum S of its current
 * state, reduced in FP64 on the device.  Per world FLP_BATCH_NSTAT doubles:
 *   0 sum S   1 sum of S > 0   2,3 centre of mass (x, y) of S > 0 (grid centre
 *   when that sum <= 1e-6)   4 radius (second moment about it)
 *   5 max(0, max S)   6 #(S > 1e-6)   7 #(S < 0)   8 mean   9 variance
 *   10 mean |S - left| + |S - up| over 2N (no wrap)   11 N. */
#define FLP_BATCH_NSTAT 12
FLP_API int flp_batch_stats(flp_batch* b, double* out, size_t n);
/* Device snapshots of every world's channel sum: reserve n_slots slots (kept
 * across calls), copy the current state's channel sums into a slot, and the
 * normalised dot product of two slots per world (0 when a norm <= 1e-6). */
FLP_API int flp_batch_reserve_snapshots(flp_batch* b, int n_slots);
FLP_API int flp_batch_snapshot(flp_batch* b, int slot);
FLP_API int flp_batch_similarity(flp_batch* b, int slot_a, int slot_b, double* out, int n);
/* As flp_profile_run: 5 stages (r2c, cols, c2r, flow, gather); stage_ms may be NULL
 * (whole steps timed only). */
FLP_API int flp_batch_profile_run(flp_batch* b, int steps, int flush_l2, float* stage_ms, float* step_ms);

/* ---- Differentiable step (adjoint) ------------------------------------
 * No counterpart in the reference (its propagators are forward only).  A
 * batch of same-shape 2D worlds -- equal width, height, channels (<= 8),
 * kernel count, per-kernel source/target channels and distribution_size;
 * every other parameter may differ per world -- run forward T steps keeping
 * the state every k steps, then a hand-written reverse sweep (recomputing
 * each k-step segment from its checkpoint) turns dL/dA_T into dL/dA_0 and
 * dL/d(parameters).  The forward pass is bit-identical to flp_run on each
 * world.  Host buffers hold all worlds back to back, world-major, each world
 * [channel][y][x].  The parameter vector of one world is
 *   beta_a, then per kernel: weight, mu, sigma, then per ring of that
 *   kernel: amplitude, distance, width
 * and the worlds' vectors are concatenated in world order. */
typedef struct flp_adjoint flp_adjoint;

FLP_API int flp_adj_create(const char* const* config_jsons, int n_worlds, flp_adjoint** out);
FLP_API int flp_adj_destroy(flp_adjoint* h);
/* Initial state A_0 of one world (channels*W*H floats, host memory). */
FLP_API int flp_adj_write_state(flp_adjoint* h, int world, const float* state, size_t n);
FLP_API int flp_adj_state_from_seed(flp_adjoint* h, int world, const char* seed_json);
/* T steps from A_0, keeping A_0, A_k, A_2k, ... on the device. */
FLP_API int flp_adj_forward(flp_adjoint* h, int steps, int checkpoint_every);
/* A_T of one world after flp_adj_forward. */
FLP_API int flp_adj_read_final(flp_adjoint* h, int world, float* out, size_t n);
FLP_API int flp_adj_param_count(flp_adjoint* h, int world, int* count);
/* dl_dfinal: dL/dA_T of all worlds (n = n_worlds*channels*W*H floats);
 * dl_dinitial (same size) and dl_dparams (sum of the param counts) receive
 * the gradients; either may be NULL. */
FLP_API int flp_adj_backward(flp_adjoint* h, const float* dl_dfinal, size_t n, float* dl_dinitial, size_t n_initial,
                             double* dl_dparams, size_t n_params);
/* Device time of the last forward and backward passes (CUDA events). */
FLP_API int flp_adj_timings(flp_adjoint* h, float* forward_ms, float* backward_ms);

/* ---- Animation recording ------------------------------------------------
 * AnimationRecorder (src/animation/recorder.rs:56-200) for a single-world
 * handle: FLWA files (src/animation/format.rs: 52-byte header, raw f32
 * little-endian frames of all channels, a 16-byte index entry per frame at
 * the end) that the reference's AnimationPlayer reads.  Recording does not
 * stall the handle's stream: a frame is a device copy of the state enqueued
 * after the steps enqueued so far, moved to pinned host memory on a separate
 * stream and written by a writer thread; flp_rec_record blocks only while all
 * 4 frame slots are in flight.  compression: 0 = none; 1 (LZ4) is refused
 * with FLP_ERR_UNSUPPORTED, as the reference refuses it without its optional
 * lz4 feature.  The handle must outlive the recorder. */
typedef struct flp_recorder flp_recorder;

/* AnimationRecorder::new: creates the file and writes a placeholder header.
 * frame_skip >= 1 records every frame_skip-th call; max_frames 0 = unlimited. */
FLP_API int flp_rec_create(flp_propagator* h, const char* path, int compression, uint32_t frame_skip,
                           uint64_t max_frames, flp_recorder** out);
/* record_frame (recorder.rs:109-166) of the handle's current state, in stream
 * order; *recorded (may be NULL) says whether this call took a frame. */
FLP_API int flp_rec_record(flp_recorder* r, int* recorded);
/* `steps` times: one step of the handle, then flp_rec_record. */
FLP_API int flp_rec_run(flp_recorder* r, uint64_t steps);
FLP_API int flp_rec_frames_written(flp_recorder* r, uint64_t* n);
/* finalize (recorder.rs:171-200): waits for the frames in flight, appends the
 * index table, rewrites the header with the frame count, closes the file and
 * frees the recorder; the outputs (may be NULL) are AnimationStats' fields. */
FLP_API int flp_rec_finalize(flp_recorder* r, uint64_t* frame_count, uint64_t* total_bytes,
                             uint64_t* avg_frame_bytes);

/* ---- Parameter-embedded worlds -----------------------------------------
 * EmbeddedPropagator (src/compute/embedded_propagator.rs:144-345): a 2D world
 * whose cells carry their own CellParams {mu, sigma, weight, beta_a, n}
 * (src/schema/embedding.rs:20-31) that are advected and mixed with the mass.
 * The config's "embedding" object is EmbeddingConfig {enabled,
 * mixing_temperature, linear_mixing} (embedding.rs:331-352).  Parameter grids
 * cross the ABI as channels*cells*5 floats, cell-major with the 5 fields in
 * struct order (ParameterGrid's layout, embedding.rs:178-186).  Kernel radii
 * up to 64 cells; 3D configs are rejected with FLP_ERR_UNSUPPORTED. */
typedef struct flp_embedded flp_embedded;

/* EmbeddedPropagator::new (embedded_propagator.rs:177-221); the state starts
 * at zero mass with EmbeddedState::from_seed's parameters. */
FLP_API int flp_emb_create(const char* config_json, flp_embedded** out);
FLP_API int flp_emb_destroy(flp_embedded* h);
/* EmbeddedState::from_seed (embedded_propagator.rs:41-69): the seed's
 * channels, every cell at the first kernel's mu/sigma/weight and the flow's
 * beta_a/n; time and step reset to 0. */
FLP_API int flp_emb_state_from_seed(flp_embedded* h, const char* seed_json);
/* Replace the state (channels*cells floats) and, when params is not NULL,
 * its parameter grids (channels*cells*5 floats); both copied in. */
FLP_API int flp_emb_write_state(flp_embedded* h, const float* channels, size_t n, const float* params,
                                size_t n_params, float time, uint64_t step);
/* Copy the state out; channels, params, time and step may each be NULL. */
FLP_API int flp_emb_read_state(flp_embedded* h, float* channels, size_t n, float* params, size_t n_params,
                               float* time, uint64_t* step);
/* EmbeddedPropagator::step / run (embedded_propagator.rs:222-345), on the
 * handle's stream; run replays a captured CUDA graph.  Asynchronous. */
FLP_API int flp_emb_step(flp_embedded* h);
FLP_API int flp_emb_run(flp_embedded* h, uint64_t n);
/* Wait for the stream; FLP_ERR_NONFINITE when a non-finite mass was seen. */
FLP_API int flp_emb_synchronize(flp_embedded* h);
/* FP64 compensated total mass of all channels. */
FLP_API int flp_emb_total_mass(flp_embedded* h, double* out);
/* Device time of `steps` steps (CUDA events around flp_emb_run).  With
 * stage_ms (3 floats) the steps run one by one with events between the
 * kernels: convolution + growth, flow, gather (totals over the steps). */
FLP_API int flp_emb_profile_run(flp_embedded* h, uint64_t steps, float* step_ms, float* stage_ms);
FLP_API void* flp_emb_stream(flp_embedded* h);

/* Allocation-free affinity.  No counterpart in the reference: an addition for
 * callers that may not allocate device memory, such as code enqueued from
 * another framework's plugin or custom operator on that framework's stream,
 * where cudaMalloc would synchronise the device and fragment the memory pool
 * that the framework manages.  Computes the same
 * affinity as the direct path of flp_debug_affinity -- U = sum_k w_k
 * G(K_k * A_src) for a 2D config -- from the caller's device state
 * (channels*N floats) into the caller's device buffer d_affinity
 * (channels*N floats), on `stream` (NULL = the default stream).  The kernel
 * descriptors and stencil taps go into a 1 MiB file-scope device array, held
 * on every device that loads the library until exit; configs whose taps do
 * not fit, or with a kernel radius above 24, are rejected with
 * FLP_ERR_INVALID_ARGUMENT.  The first call on a device looks up the array's
 * device address (once per device); make that first call before any stream
 * capture.  Calls share the array, so calls that overlap on the GPU race and
 * must be serialised by the caller.  Calls no cudaMalloc or cudaFree. */
FLP_API int flp_affinity_noalloc(const char* config_json, const float* d_state, float* d_affinity, void* stream);

/* ---- Failure injection (tests of the error paths) ----------------------
 * No counterpart in the reference.  Every device allocation of the library
 * is counted; after `after` further successful allocations the next one fails
 * as if the device were out of memory (host side: the driver is not called),
 * so a test can make each allocation of flp_create, flp_batch_create,
 * flp_emb_create or flp_adj_create fail in turn and check that the call
 * returns FLP_ERR_OOM and frees what it had allocated.  after < 0 switches
 * the injection off (the default).  Process-wide; not for production use. */
FLP_API int flp_debug_fail_device_alloc(int64_t after);
/* Device allocations of the library that are currently live. */
FLP_API int flp_debug_live_device_allocs(int64_t* live);

#ifdef __cplusplus
}
#endif

#endif /* FLOWLENIA_CUDA_H */
