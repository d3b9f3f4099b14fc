/*
 * ctb200.h — C ABI of libctb200.so, the B200 (sm_100a) backend for
 * QtCTReconstruction's parallel-beam FBP path.
 *
 * Every entry point uses plain pointers, sizes and integer status codes: no C++
 * or torch types cross this boundary and no exception escapes it. Host
 * pointers are caller-owned; device workspaces are owned by the context.
 * A context serialises its own calls with an internal mutex, so one context
 * may be shared by threads (the reference controller calls computeSinogram
 * from an OpenMP loop, CtReconstructionController.cpp:1232-1242).
 *
 * Conventions follow the reference's SerialBackend (the oracle):
 *   slice        [y][x] row-major float, width x height   (CTTypes.h:15-74)
 *   volume       [z][y][x] float                          (CTTypes.h:101)
 *   sinogram     [angle][bin] float, na rows of nd bins   (SerialBackend.cpp:82-83)
 *   sinograms    [z][angle][bin]  (the consumer volume (nz, na, bins))
 *   angles       degrees, float; uniform angles are 180/na * a in float
 *   filter ids   ReconstructionParams::FilterType order   (CTTypes.h:151)
 *
 * Citations name files of the QtCTReconstruction project.
 */
#ifndef CTB200_H
#define CTB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ctb_ctx ctb_ctx;

typedef enum ctb_status {
    CTB_OK = 0,
    CTB_ERR_INVALID = 1,      /* bad sizes or null pointers (reference: empty result) */
    CTB_ERR_CUDA = 2,         /* a CUDA runtime call failed; see ctb_last_error */
    CTB_ERR_OOM = 3,          /* device allocation failed or budget exceeded */
    CTB_ERR_UNSUPPORTED = 4,  /* size outside what the kernels support */
    CTB_ERR_NO_DEVICE = 5,    /* no usable sm_100 device */
    CTB_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up */
    CTB_ERR_CANCELLED = 7,    /* serving: request cancelled */
    CTB_ERR_NOT_FOUND = 8,    /* serving: unknown request id */
    CTB_ERR_BUSY = 9          /* serving: request still running */
} ctb_status;

/* ReconstructionParams::FilterType (CTTypes.h:151). */
typedef enum ctb_filter {
    CTB_FILTER_RAMP = 0,
    CTB_FILTER_SHEPP_LOGAN = 1,
    CTB_FILTER_HAMMING = 2,
    CTB_FILTER_COSINE = 3,
    CTB_FILTER_HANN = 4,
    CTB_FILTER_BARTLETT = 5
} ctb_filter;

/* Output units of a reconstruction from sinograms.
 *   NONE    normalised units, as SerialBackend::reconstructSlice returns them
 *           (SerialBackend.cpp:142-255) and as the interface's default
 *           reconstructVolumeFromSinograms stores them (BackendFactory.cpp:17-60);
 *   SERIAL  out * (span <= 0 ? 1 : span) + min   (SerialBackend.cpp:297-304);
 *   OPENMP  out * span + min, or min everywhere when span <= 0
 *           (OpenMPBackend.cpp:37-59).
 * min/span come from the per-slice stats (see ctb_forward_d). */
typedef enum ctb_denorm {
    CTB_DENORM_NONE = 0,
    CTB_DENORM_SERIAL = 1,
    CTB_DENORM_OPENMP = 2,
    CTB_DENORM_CUDA = 3   /* out * span + min when span > 0, else out (CUDABackend.cu:676-681) */
} ctb_denorm;

/* ---------------------------------------------------------------- lifecycle */

/* Create a context on CUDA device `device`. Replaces the construction done by
 * BackendFactory::create (BackendFactory.cpp:62-82); CTB_ERR_NO_DEVICE is the
 * isAvailable() == false case (IReconstructionBackend.h:18). */
ctb_status ctb_create(ctb_ctx** out, int device);
void ctb_destroy(ctb_ctx* ctx);
/* Message of the last failure on this context ("" if none). */
const char* ctb_last_error(const ctb_ctx* ctx);
const char* ctb_status_string(ctb_status s);
/* Run subsequent device work on `stream` (a cudaStream_t; NULL = the
 * context's own stream). */
ctb_status ctb_set_stream(ctb_ctx* ctx, void* stream);
/* Block until all work issued by the context has finished. */
ctb_status ctb_synchronize(ctb_ctx* ctx);
/* IReconstructionBackend::lastSinogramTimeMs / lastReconstructionTimeMs
 * (IReconstructionBackend.h:50-54): device time of the last forward and
 * filter+backprojection stages, measured with CUDA events. */
double ctb_last_sinogram_ms(const ctb_ctx* ctx);
double ctb_last_reconstruction_ms(const ctb_ctx* ctx);
/* Device time of the last summed-ellipsoid phantom kernel (ctb_phantom_sum[_d]),
 * CUDA events around its launch; no counterpart in the reference. */
double ctb_last_phantom_ms(const ctb_ctx* ctx);
/* Number of kernel launches the context has issued so far. */
uint64_t ctb_launch_count(const ctb_ctx* ctx);

/* Per-stage device timing. With profiling on, every volume reconstruction
 * (ctb_reconstruct_volume[_d]) records CUDA events between its stages into a
 * ring of 256 entries. ctb_stage_times(ctx, back, ms) reads the entry `back`
 * calls ago (0 = latest; waits for it) into ms[0..3] = {statistics +
 * normalisation, forward projection, filtering, backprojection}. */
ctb_status ctb_set_profiling(ctb_ctx* ctx, int enable);
ctb_status ctb_stage_times(ctb_ctx* ctx, int back, double* ms);
/* Device ms of the filter stage's main kernel alone in the same profiled call
 * (the FFT kernel, or the tensor-core product without its operand split). */
ctb_status ctb_filter_kernel_ms(ctb_ctx* ctx, int back, double* ms);

/* Filter implementation of the context's filter stages (ctb_reconstruct_*,
 * ctb_fbp*, the _d variants; batches and the serving loop always use the FFT):
 *   FFT         the radix-16 shared-memory FFT convolution in FP32 (default);
 *   TC_BF16X3   the same linear operator as a dense Toeplitz-matrix product on
 *               the tcgen05 tensor cores, both factors split into three BF16
 *               terms (about 24 significant bits), the six products whose
 *               terms' orders add up to at most 2 accumulated in FP32 (the
 *               dropped ones are about 2^-24 relative).
 * The reference filters with its own radix-2 FFT (FFT.cpp:9-158). */
enum { CTB_FILTER_MODE_FFT = 0, CTB_FILTER_MODE_TC_BF16X3 = 1 };
ctb_status ctb_set_filter_mode(ctb_ctx* ctx, int mode);

/* Backprojection tile shapes. Six are compiled: 0 = 32x32 voxels, 4 per
 * thread (the general case); 1 = 64x32, 8 per thread; 2 = 32x16, 2 per
 * thread; 3 = 16x16, 1 per thread; all with 32 angles per staged chunk; and
 * the 32x32 tile with 16 (4) and 64 (5) angles per chunk, which sum every
 * voxel's angles in the same order as shape 0 and so give its result bit for
 * bit. Without tuning a job gets a shape from its size alone (32x32 once its
 * tiles x slice groups reach the SM count, 32x16 above a quarter of it, else
 * 16x16). With the autotuner
 * on, the first job of each size bucket {ceil(n / 64), ceil(angles / 180),
 * floor(log2(ceil(depth / 4)))} times every shape on its own data (that call
 * synchronises) and the fastest is kept for the bucket; batches use a tuned
 * shape when their job's bucket is tuned, else the default, so a job's shape
 * never depends on the rest of a batch. The tuned table can be read and
 * loaded as int quadruples {n bucket, angle bucket, depth bucket, shape}.
 * Shapes differ in rounding only (all within the parity tolerance); no
 * counterpart in the reference. */
ctb_status ctb_set_bp_shape(ctb_ctx* ctx, int variant);  /* force a shape; -1 = automatic */
ctb_status ctb_bp_shape_info(int variant, int* tile_x, int* tile_y, int* voxels_per_thread,
                             int* angles_per_chunk);
ctb_status ctb_bp_shape_for(ctb_ctx* ctx, int output_size, int depth, int num_angles, int* variant);
ctb_status ctb_set_autotune(ctb_ctx* ctx, int enable);
ctb_status ctb_autotune_table(ctb_ctx* ctx, int* entries, int capacity, int* count);
ctb_status ctb_autotune_load(ctb_ctx* ctx, const int* entries, int count);

/* Conventions of a context's host- and device-buffer entry points (batches
 * and the serving loop always use SerialBackend's):
 *   SERIAL  SerialBackend's (the default; the oracle): pixel splat forward
 *           projector with zero pixels skipped, dropped Nyquist bin,
 *           floor(n/2) / floor(sq/2) centres, both taps required;
 *   CUDA    the reference's CUDA backend (CUDABackend.cu): every pixel
 *           normalised, ray-march bilinear forward projector with detector
 *           centre (nd-1)/2 for slices and floor(nd/2) for volumes
 *           (:108-153, :534, :759), cuFFT-style filter keeping the Nyquist bin
 *           (:603-652), backprojection with (n-1)/2 and (sq-1)/2 centres and
 *           per-tap bounds (:184-236, :672), denormalisation only when
 *           max > min (:676-681). */
enum { CTB_CONVENTION_SERIAL = 0, CTB_CONVENTION_CUDA = 1 };
ctb_status ctb_set_convention(ctb_ctx* ctx, int convention);

/* Forward projector bounds (SerialBackend convention; on by default). The
 * reference skips background pixels (SerialBackend.cpp:104-106). Here every
 * pixel whose normalised value is zero is an exact zero contribution, so the
 * projector walks each 8-slice group only where its strips of detector bins
 * meet the bounding box, the centred disc and the per-8-row-band column ranges
 * of the group's non-zero pixels.
 * enable = 0 walks the whole image (same results; for timing comparisons). */
ctb_status ctb_set_forward_bounds(ctb_ctx* ctx, int enable);

/* Measured shared-memory load bandwidth of this GPU in GB/s: a conflict-free
 * 16-byte-per-lane load loop over all SMs, timed with CUDA events. The
 * backprojector's roofline denominator. */
ctb_status ctb_probe_smem_bandwidth(ctb_ctx* ctx, double* gbs);

/* Diagnostics. The reference reports device failures by printing or throwing
 * (CUDABackend.cu:37-43, HybridBackend.cu:44-65); here every device-side wait
 * is bounded (2 s of the GPU's global timer) and a wait that gives up makes
 * the call return CTB_ERR_TIMEOUT with the context still usable.
 * ctb_selftest_bounded_wait runs that path on purpose: one CTA waits, at most
 * `limit_us` microseconds (1 .. 2e6), on a barrier that nothing completes (no
 * copy is in flight), records the timeout and returns. It returns
 * CTB_ERR_TIMEOUT when the path works (CTB_OK would mean the wait was not
 * bounded).
 * ctb_set_fault_injection (host side, for tests): with slab >= 0 the next
 * ctb_reconstruct_volume calls fail with CTB_ERR_CUDA after queuing that
 * slab's copy and forward stage, with earlier slabs still in flight; such a
 * failed call returns only after all its copies and kernels have finished.
 * -1 (the default) turns it off. */
ctb_status ctb_selftest_bounded_wait(ctb_ctx* ctx, unsigned limit_us);
ctb_status ctb_set_fault_injection(ctb_ctx* ctx, int slab);

/* Geometry helpers shared with the reference (SerialBackend.cpp:152-163):
 * square_bins = ceil(sqrt(2)*bins), pad_before = square_bins/2 - bins/2,
 * fft_size = max(64, nextPow2(2*square_bins)). */
ctb_status ctb_pad_geometry(int bins, int* square_bins, int* pad_before, int* fft_size);
/* FilterDesign::createFilter (FilterDesign.cpp:13-111), evaluated in double
 * precision and rounded to float: fft_size/2+1 values. */
ctb_status ctb_filter_response(int fft_size, int filter, float* H);

/* ------------------------------------------- host-buffer entry points
 * These mirror IReconstructionBackend (IReconstructionBackend.h:10-55); the
 * B200Backend C++ class forwards to them. Host<->device copies are inside. */

/* IReconstructionBackend::computeSinogram (SerialBackend.cpp:59-136).
 * sino_out: num_angles x detector_bins. angles_deg_out (num_angles) and
 * minmax_out {min, max} may be NULL. */
ctb_status ctb_compute_sinogram(ctb_ctx* ctx, const float* slice, int width, int height,
                                int num_angles, int detector_bins, float* sino_out,
                                float* angles_deg_out, float* minmax_out);

/* IReconstructionBackend::reconstructSlice (SerialBackend.cpp:142-255):
 * normalised units, output_size x output_size. */
ctb_status ctb_reconstruct_slice(ctb_ctx* ctx, const float* sino, int num_angles,
                                 int detector_bins, const float* angles_deg, int output_size,
                                 int filter, float* out);
/* reconstructSlice with the Sinogram's original_min_hu / original_max_hu: the
 * CUDA convention denormalises with them when max > min (CUDABackend.cu:
 * 676-681); the Serial convention ignores them (normalised units, as
 * SerialBackend::reconstructSlice). ctb_reconstruct_slice = min = max = 0. */
ctb_status ctb_reconstruct_slice_hu(ctb_ctx* ctx, const float* sino, int num_angles, int detector_bins,
                                    const float* angles_deg, int output_size, int filter, float min_hu,
                                    float max_hu, float* out);

/* IReconstructionBackend::reconstructVolume (SerialBackend.cpp:261-318):
 * per slice, forward projection onto detector_bins bins (the reference passes
 * detector_bins = n), FBP back to n x n and denormalisation with the slice's
 * min/span. vol and out: depth x n x n. */
ctb_status ctb_reconstruct_volume(ctb_ctx* ctx, const float* vol, int n, int depth,
                                  int num_angles, int detector_bins, int filter, float* out);

/* IReconstructionBackend::reconstructVolumeFromSinograms
 * (IReconstructionBackend.h:39-44; default loop BackendFactory.cpp:17-60).
 * sinos: depth x num_angles x bins; out: depth x bins x bins. The per-slice
 * min/max used by SERIAL/OPENMP denormalisation are taken from the sinogram
 * itself, as the reference's default implementation does. */
ctb_status ctb_reconstruct_from_sinograms(ctb_ctx* ctx, const float* sinos, int depth,
                                          int num_angles, int bins, const float* angles_deg,
                                          int filter, int denorm, float* out);

/* ------------------------------------------- device-buffer entry points
 * Inputs already resident in device memory; work is queued on the context's
 * stream and the call returns without synchronising. */

/* Forward projection of depth slices (n x n each) to sinograms
 * d_sino[z][a][detector_bins]. d_stats receives 4 floats per slice:
 * {min, max, span_fwd, span_denorm} with span_fwd = (max-min < 1e-6 ? 1 : max-min)
 * (SerialBackend.cpp:78-80) and span_denorm = (max-min <= 0 ? 1 : max-min)
 * (SerialBackend.cpp:298-300). angles_deg: host array (NULL = uniform). */
ctb_status ctb_forward_d(ctb_ctx* ctx, const float* d_vol, int n, int depth, int num_angles,
                         int detector_bins, const float* angles_deg, float* d_sino,
                         float* d_stats);

/* Ramp filtering + backprojection of d_sino[z][a][bins] into
 * d_out[z][output_size][output_size]. d_stats (4 floats per slice, as written
 * by ctb_forward_d) selects the denormalisation; NULL means normalised units. */
ctb_status ctb_fbp_d(ctb_ctx* ctx, const float* d_sino, int depth, int num_angles, int bins,
                     const float* angles_deg, int output_size, int filter, const float* d_stats,
                     int denorm, float* d_out);

/* Filtering (any CTB_FILTER_* id; others return CTB_ERR_INVALID) +
 * backprojection of 1..4 slices that allocates no device
 * memory; it has no counterpart in the reference. It exists for callers that
 * cannot allocate device memory where they reconstruct (a caller-owned memory
 * pool, a real-time loop that must not wait on an allocator, a host whose
 * allocator is not cudaMalloc) and so cannot create a context, whose
 * workspaces are allocated on demand. The caller passes device buffers
 * d_sino[depth][num_angles][bins] and d_out[depth][output_size]^2; the result
 * is in normalised units (no denormalisation: the same values as ctb_fbp_d
 * with d_stats = NULL and as SerialBackend::reconstructSlice), and the call
 * returns after `stream` (a cudaStream_t, NULL = legacy default stream) has
 * finished it. Every intermediate lives in one static 16 MiB device array that
 * each GPU using the library keeps until the process exits: at most 2048
 * angles, convolution length nextPow2(square_bins + bins - 1) <= 8192 and
 * num_angles x (filtered row pitch) within the array; larger requests return
 * CTB_ERR_UNSUPPORTED. The first call on a device looks up the array's device
 * address (make it before any stream capture). All calls share the array, so
 * calls that overlap on the GPU race. */
ctb_status ctb_fbp_noalloc(const float* d_sino, int depth, int num_angles, int bins,
                           const float* angles_deg, int output_size, int filter, float* d_out,
                           void* stream);

/* reconstructVolume on device buffers: forward + filter + backprojection +
 * Serial denormalisation. */
ctb_status ctb_reconstruct_volume_d(ctb_ctx* ctx, const float* d_vol, int n, int depth,
                                    int num_angles, int detector_bins, int filter, float* d_out);

/* ------------------------------------------------------------ batches */

/* One FBP job of a batch: ramp filtering + backprojection of device sinograms
 * sino[depth][num_angles][bins] into out[depth][output_size]^2, in normalised
 * units (ctb_fbp_d with d_stats = NULL). angles_deg is a host array read when
 * the batch is created (NULL = uniform 180/na * a). No counterpart in the
 * reference, which reconstructs one volume per call
 * (IReconstructionBackend.h:39-44); a job's result is bit-identical to
 * ctb_fbp_d on the same job and does not depend on the other jobs. */
typedef struct ctb_fbp_job {
    const float* sino;
    int depth;
    int num_angles;
    int bins;
    const float* angles_deg;
    int output_size;
    int filter;
    float* out;
} ctb_fbp_job;

typedef struct ctb_batch ctb_batch;

enum {
    CTB_BATCH_GRAPH = 1,    /* capture the launches once as a CUDA graph; ctb_batch_run replays it */
    CTB_BATCH_PER_JOB = 2,  /* one filter + one backprojection launch per job (comparison mode) */
    CTB_BATCH_PERSISTENT = 4 /* backprojection on a persistent grid drawing (job, slice group, tile)
                                items from an atomic counter instead of one CTA per item */
};

/* Plan a batch: device state for every job (angle tables, filtered rows) is
 * allocated here, jobs are grouped by convolution length, and the work of all
 * jobs shares one filter launch per length class and one backprojection launch
 * per tile shape over the (job, slice group, tile) items, longest jobs first
 * (one CTA per item by default, a persistent work queue with
 * CTB_BATCH_PERSISTENT). The batch keeps the job pointers; it must be
 * destroyed before its context. */
ctb_status ctb_batch_create(ctb_ctx* ctx, const ctb_fbp_job* jobs, int njobs, int flags,
                            ctb_batch** out);
/* Enqueue the batch on the context's stream (asynchronous). */
ctb_status ctb_batch_run(ctb_batch* batch);
/* Kernel launches (or graph launches) one ctb_batch_run issues; voxel-angle
 * updates of the whole batch (sum of output_size^2 * depth * num_angles). */
ctb_status ctb_batch_info(const ctb_batch* batch, int* launches, double* updates,
                          size_t* device_bytes);
void ctb_batch_destroy(ctb_batch* batch);

/* ctb_batch_create + run + synchronise + destroy. */
ctb_status ctb_fbp_batch_d(ctb_ctx* ctx, const ctb_fbp_job* jobs, int njobs);

/* Plain one-request-per-call FBP on host buffers: sinos[depth][na][bins] are
 * filtered and backprojected into out[depth][output_size]^2 (normalised
 * units); returns when done. The stack is streamed in slabs of slices: the
 * next slab's sinograms copy in and the previous slab's slices copy out on
 * their own streams while the current slab is computed (the reference's CUDA
 * backend likewise pipelines pinned copies on two streams, CUDABackend.cu:
 * 370-452,739-863). Copies overlap fully only from page-locked host memory.
 * The result equals one pass over the whole stack bit for bit. The
 * reference's reconstructVolumeFromSinograms with an explicit output size
 * (BackendFactory.cpp:17-60 reconstructs slice by slice);
 * ctb_reconstruct_from_sinograms runs the same pipeline. */
ctb_status ctb_fbp(ctb_ctx* ctx, const float* sinos, int depth, int num_angles, int bins,
                   const float* angles_deg, int output_size, int filter, float* out);

/* ------------------------------------------------------------ serving */

/* A serving loop on one GPU (no counterpart in the reference). Requests of
 * different sizes, angle counts and filters are submitted at any time; a
 * scheduler thread admits them in arrival order while their device footprint
 * (sinograms, angle table, filtered rows, volume) fits the memory budget, copy
 * threads move host data on their own streams (directly from page-locked
 * memory, else through pinned staging buffers), and every scheduling
 * iteration packs the requests whose data is on the device into one batch
 * (ctb_batch semantics: one filter launch per convolution length, one
 * backprojection launch per tile shape over all the batch's (request, slice
 * group, tile) items) while other requests upload and download. Results are
 * bit-identical to ctb_fbp_d on the same request. */
typedef struct ctb_server ctb_server;

typedef struct ctb_server_config {
    int device;
    size_t memory_budget;  /* device bytes for request state; 0 = min(120 GB, 85% of free) */
    int max_batch;         /* requests per batch, 1..64; 0 = 64 */
    int copy_threads;      /* staging threads per direction; 0 = 4 */
    size_t staging_bytes;  /* pinned staging per copy thread; 0 = 64 MiB */
    int fault_every;       /* > 0: every fault_every-th request fails its upload with
                              CTB_ERR_CUDA (host-side fault injection for tests); 0 = off */
} ctb_server_config;

enum { CTB_REQ_DEVICE = 1 /* sino and out are device pointers: nothing is staged */ };

typedef struct ctb_request {
    const float* sino;        /* [depth][num_angles][bins], host unless CTB_REQ_DEVICE */
    int depth;
    int num_angles;
    int bins;
    const float* angles_deg;  /* host, copied at submit; NULL = uniform 180/na * a */
    int output_size;
    int filter;
    float* out;               /* [depth][output_size]^2, host unless CTB_REQ_DEVICE */
    int flags;
} ctb_request;

typedef struct ctb_server_stats {
    uint64_t submitted, completed, failed, cancelled, rejected;
    uint64_t batches;         /* batch launches */
    double mean_batch;        /* requests per batch */
    double p50_ms, p99_ms, max_ms;  /* submit-to-done latency of completed requests */
    double volumes_per_s;     /* completed / (last completion - first submission) */
    double updates_per_s;     /* voxel-angle updates of completed requests over the same span */
    size_t memory_budget, memory_peak;
} ctb_server_stats;

ctb_status ctb_server_create(const ctb_server_config* config, ctb_server** out);
/* Queue a request; *id identifies it. A request whose footprint exceeds the
 * budget is rejected with CTB_ERR_OOM. The host buffers must stay valid until
 * the request is final. */
ctb_status ctb_server_submit(ctb_server* s, const ctb_request* req, uint64_t* id);
/* CTB_OK when done, CTB_ERR_BUSY while queued or running, the request's error
 * status if it failed or was cancelled, CTB_ERR_NOT_FOUND for unknown ids. */
ctb_status ctb_server_poll(ctb_server* s, uint64_t id);
/* As poll, waiting up to timeout_ms (< 0: no limit). */
ctb_status ctb_server_wait(ctb_server* s, uint64_t id, double timeout_ms);
/* Cancel a request: a queued one never runs; a running one finishes on the
 * device but its result is not copied out. Final status CTB_ERR_CANCELLED. */
ctb_status ctb_server_cancel(ctb_server* s, uint64_t id);
/* Forget a final request (its id becomes unknown). */
ctb_status ctb_server_release(ctb_server* s, uint64_t id);
ctb_status ctb_server_get_stats(ctb_server* s, ctb_server_stats* out);
/* Waits for running work, cancels queued requests, frees everything. */
void ctb_server_destroy(ctb_server* s);

/* The server's admission allocator, usable on its own (host bookkeeping only,
 * no device calls): first fit over [0, capacity) in 256-byte units, adjacent
 * free ranges merged. */
typedef struct ctb_arena ctb_arena;
ctb_status ctb_arena_create(size_t capacity, ctb_arena** out);
ctb_status ctb_arena_alloc(ctb_arena* a, size_t bytes, size_t* offset);  /* CTB_ERR_OOM if no fit */
ctb_status ctb_arena_free(ctb_arena* a, size_t offset);                  /* CTB_ERR_NOT_FOUND */
ctb_status ctb_arena_stats(const ctb_arena* a, size_t* used, size_t* peak, size_t* largest_free);
void ctb_arena_destroy(ctb_arena* a);

/* ------------------------------------------------------- sinogram files */

/* The consumer format of the reference: sinograms as an NPY array
 * (depth, num_angles, bins) of little-endian float32 plus a sidecar
 * "<name>.meta.json" {version, depth, num_angles, detector_bins,
 * detector_spacing_mm, original_min_hu, original_max_hu, angles_deg}
 * (CtReconstructionController.cpp:1353-1482 export, :1494-1616 import; NPY
 * layout FileIO.cpp:53-148). Host-only, no device calls.
 *
 * ctb_sinogram_file_shape reads the NPY header (versions 1-3, '<f4', C order,
 * three dimensions) without the data. ctb_load_sinogram_file reads the data
 * into sinos (depth * num_angles * bins floats) and, when non-NULL, the angles
 * (num_angles floats: the sidecar's when their count is num_angles, else
 * uniform 180/na * a) and meta[3] = {detector_spacing_mm (default 1),
 * min, max (the sidecar's, else computed from the data)}.
 * ctb_save_sinogram_file writes both files (angles NULL = uniform). */
ctb_status ctb_sinogram_file_shape(const char* path, int* depth, int* num_angles, int* bins);
ctb_status ctb_load_sinogram_file(const char* path, float* sinos, float* angles_deg, float* meta);
ctb_status ctb_save_sinogram_file(const char* path, const float* sinos, int depth, int num_angles, int bins,
                                  const float* angles_deg, float spacing_mm, float min_hu, float max_hu);

/* ------------------------------------------------------------ phantoms */

/* Summed random-ellipsoid phantom (the benchmark phantom; a new generator mode
 * beside Generator3D). Records of 16 floats per ellipsoid: centre (3),
 * rotation rows (9), inverse squared semi-axes (3), density (1); voxel
 * coordinates (2i-(n-1))/n per axis, zero outside the unit sphere. */
ctb_status ctb_phantom_params(uint64_t seed, int count, float* params);
ctb_status ctb_phantom_sum_d(ctb_ctx* ctx, const float* params, int count, int nx, int ny,
                             int nz, float* d_vol);
ctb_status ctb_phantom_sum(ctb_ctx* ctx, const float* params, int count, int nx, int ny, int nz,
                           float* vol);

/* Generator3D::generateBrainHU on the GPU with the CPU generator's random
 * stream (Generator3DCPU.cpp:35-117): axis-aligned ellipsoids in millimetres,
 * max-composited over -1000 HU. tissue: soft then bone tissue, 8 floats each
 * {hu_min, hu_max, size_min_mm, size_max_mm, peripheral_only, r_min, r_max,
 * probability} (Generator3D.h:16-34). */
ctb_status ctb_generator3d(ctb_ctx* ctx, int nx, int ny, int nz, float radius_mm, int count,
                           uint32_t seed, const float* tissue, float* vol);

/* --------------------------------------------------------- point cloud */

/* IReconstructionBackend::extractPointCloud (SerialBackend.cpp:325-346) with
 * index coordinates: points (x, y, z, hu) with hu > threshold in z, y, x
 * order. Writes at most `capacity` points; *count receives the total. */
ctb_status ctb_extract_point_cloud(ctb_ctx* ctx, const float* vol, int nx, int ny, int nz,
                                   float threshold, float* points, int64_t capacity,
                                   int64_t* count);

#ifdef __cplusplus
}
#endif

#endif /* CTB200_H */
