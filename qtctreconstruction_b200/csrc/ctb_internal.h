// ctb_internal.h — shared declarations of libctb200.so (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ctb200.h"

namespace ctb {

// ----------------------------------------------------------------- geometry
// Padded detector geometry of reconstructSlice (SerialBackend.cpp:152-163).
struct PadGeom {
    int bins = 0;  // detector bins of the input sinogram
    int sq = 0;    // square_bins = ceil(sqrt(2) * bins)
    int pad = 0;   // pad_before = sq/2 - bins/2
    int L = 0;     // fft_size = max(64, nextPow2(2 * sq))
    int Lc = 0;    // convolution length used on the device: max(64, nextPow2(sq + bins - 1))
};
PadGeom pad_geometry(int bins);
// The reference filters a row by circular convolution, length L, with
// h = IDFT_L(H~) (H~[k] = H[min(k, L-k)], bins 0 and L/2 zero). Only lags
// d in [-(pad + bins - 1), sq - 1 - pad] ever meet data, a range of sq + bins - 1
// <= Lc samples, so the same linear operator is a circular convolution of length
// Lc with h restricted to those lags. With the row placed at positions [0, bins)
// of the length-Lc sequence, lag d sits at (d + pad) mod Lc and filtered bin i
// is position i. Returns DFT_Lc of that kernel divided by Lc (re, im
// interleaved), evaluated in double precision.
std::vector<double> conv_response(const PadGeom& g, int type, bool keep_nyquist = false);
// The same kernel in the lag domain: h(d) for d = -(pad + bins - 1) .. sq - 1 - pad
// (index d + pad + bins - 1), double precision. Filtered bin i of a row x is
// sum_j h(i - pad - j) x[j].
std::vector<double> conv_kernel(const PadGeom& g, int type, bool keep_nyquist = false);

// Layout of the filtered rows the backprojector reads: for each group of four
// slices and each angle, `pitch` bins of float4 (one float per slice), with
// `guard` zero bins in front of bin 0 so that every staged window lies inside
// the row.
struct FiltLayout {
    int sq = 0;
    int guard = 0;
    int pitch = 0;
};
constexpr int kBpTileMax = 64;     // widest backprojection tile edge (voxels)
constexpr int kBpWindowMax = 76;   // most bins staged per angle and tile
FiltLayout filt_layout(int sq, int n_out);

// Backprojection tile shapes ("variants"): tx x ty voxels, vpt voxels per
// thread, ca angles per staged chunk, win bins per staged window.
constexpr int kBpVariants = 6;
struct BpShape {
    int tx, ty, vpt, ca, win;
};
BpShape bp_shape(int variant);
// The shape used without tuning: a function of the job's size only.
int bp_default_variant(int n_out, int nz, int sms);

// FilterDesign (FilterDesign.cpp:13-111) in double precision: fft_size/2+1 values.
std::vector<double> filter_response(int L, int type);

// ----------------------------------------------------------- device buffer
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

// Angle tables on the device.
//   cs:  (cos, sin) in double precision of theta = deg * pi / 180 (sincospi),
//        the values every interpolation weight is computed from;
//   csf: the reference's own float (cos, sin) of degToRad(deg) (Utils.cpp:44-46
//        with libm cosf/sinf), used only to reproduce its discontinuous
//        decisions (which taps exist at the detector edges) bit for bit.
struct Trig {
    const double2* cs = nullptr;
    const float2* csf = nullptr;
};

// Kernel launchers (implemented in the .cu files). Each returns the CUDA error
// of the launch.
cudaError_t launch_trig(const float* d_angles_deg, int na, double2* d_cs, cudaStream_t st);
cudaError_t launch_slice_stats(const float* d_vol, long long npx, int nz, float4* d_stats,
                               cudaStream_t st, int4* d_box = nullptr, int2* d_band = nullptr,
                               int nband = 0);
cudaError_t launch_normalize(const float* d_vol, int w, int h, int nz, const float4* d_stats,
                             float4* d_img, float4* d_imgT, cudaStream_t st, int skip_zero = 1,
                             int4* d_box = nullptr, int2* d_band = nullptr);
// The reference CUDA backend's ray-march forward projector over the
// normalised image planes (img only).
cudaError_t launch_raymarch(const float4* d_img, int w, int h, int nz, int na, int nd, float det_center,
                            const double2* d_cs, float* d_sino, cudaStream_t st);
// Forward projector work plan: angles grouped (up to kFwdGroup per CTA, in
// their given order) by walked axis, so that the angles of a CTA read the
// same image rows at the same time. groups: {first index into order, count,
// axis (0 rows, 1 columns), K}, K the output bins per strip of the group
// (fwd_strip_bins of its smallest |kq|); max_strips = ceil(nd / smallest K).
constexpr int kFwdRows = 16;   // walked rows per chunk (crossing in double once per chunk)
constexpr int kFwdGroup = 4;   // angles per CTA
constexpr int kFwdPlanes = 2;  // float4 image planes (4 slices each) per thread
// Zero border of the normalised image planes: kFwdGuard pixels on both sides
// of every row (the projector's windows reach at most 50 columns outside the
// image) and kFwdRows rows after the last, so that every chunk the projector
// walks reads inside the plane.
constexpr int kFwdGuard = 64;
inline size_t fwd_plane_elems(int np, int nq) {
    return static_cast<size_t>(np + kFwdRows) * static_cast<size_t>(nq + 2 * kFwdGuard);
}
// Float4 planes allocated for nz slices: whole groups of kFwdPlanes, since a
// projector CTA reads all planes of its group. The kFwdPlanes = 2 planes of a
// pair are interleaved per pixel (two float4: 8 slices in 32 bytes), so a pair
// occupies 2 fwd_plane_elems float4.
inline size_t fwd_plane_count(int nz) {
    const int ng4 = (nz + 3) / 4;
    return static_cast<size_t>((ng4 + kFwdPlanes - 1) / kFwdPlanes * kFwdPlanes);
}
// Output bins per strip for a walked-axis coefficient |kq| (>= 1/sqrt 2): the
// 32 lanes of a warp hold the pixels from -1/2 |kq| to 31.5 |kq| bins above the
// strip's lower edge, which must cover the strip's K bins and the bin on
// either side: K = floor(31.5 |kq|) - 1. (A pixel just past either end, whose
// exact place the float arithmetic blurs by ~1e-6 bins, has a hat weight of
// that order on the strip's outer bins.)
inline int fwd_strip_bins(double akq) { return static_cast<int>(std::floor(31.5 * akq)) - 1; }
struct FwdPlan {
    std::vector<int> order;
    std::vector<int> groups;  // 4 ints per group
    int max_strips = 0;
};
FwdPlan forward_plan(const float* angles_deg, int na, int w, int h, int nd);
// Per-angle constants of the forward projector, in plan order (slot i holds
// angle order[i], walked along its group's axis): kq and kp, the coefficients
// of the gathered and the walked axis, inv = 1 / kq, idq = 1 / dq with
// dq = -kp inv (0 when kp = 0), the reference's float (cos, sin) and the angle
// index. Computed once per plan from the angle table, so the projector's
// per-CTA set-up reads one record instead of the order and trig tables and
// divides nothing.
struct FwdAngleRec {
    double kq, kp, inv, idq;
    float cf, sf;
    int a, pad;
};
cudaError_t launch_fwd_angles(const int4* d_groups, int ngroups, const int* d_order, Trig trig,
                              FwdAngleRec* d_rec, cudaStream_t st);
cudaError_t launch_forward(const float4* d_img, const float4* d_imgT, int w, int h, int nz,
                           int na, int nd, const int4* d_groups, int ngroups, int max_strips,
                           const FwdAngleRec* d_rec, const int4* d_box, const int2* d_band, float* d_sino,
                           cudaStream_t st);
// Twiddle tables of the filter's FFT of length L (every radix-16 pass and the
// radix-2/4/8 last pass, r-major per pass), correctly rounded from double
// precision: fft_twiddle_len(L) float2 entries; for L <= kPackedMaxL followed,
// from float2 index packed_offset(fft_twiddle_len(L)), by the same entries as
// float4 {wx, wx, wy, wy} for the packed two-sequence kernel.
constexpr int kPackedMaxL = 2048;
inline size_t packed_offset(size_t n) { return (n + 1) & ~size_t(1); }
size_t fft_twiddle_len(int L);
std::vector<float2> fft_twiddle_table(int L);
// The filter's convolution spectrum (conv_response rounded to float2, Lc
// entries); for Lc <= kPackedMaxL followed by the same values as float4
// {hx, hx, hy, hy} (Lc of them, from float2 index Lc).
std::vector<float2> filter_table(const PadGeom& g, int type, bool keep_nyquist = false);
cudaError_t launch_filter(const float* d_sino, int nz, int na, const PadGeom& g,
                          const FiltLayout& fl, const float2* d_Hc, const float2* d_tw,
                          const float4* d_stats, int denorm, float scale, float4* d_filt,
                          cudaStream_t st);

// ------------------------------------------------ tensor-core filter option
// Toeplitz filter matrix T[i][j] = h(i - pad - j) split into three BF16 terms
// (rows padded to ntiles * bn, columns to kpad), with the TMA tensor map of
// each term (opaque CUtensorMap bytes).
struct GemmTable {
    DevBuf T;
    int bn = 0, ntiles = 0, nrows = 0, kpad = 0;
    alignas(64) unsigned char map[3][128];
};
cudaError_t make_gemm_table(const PadGeom& g, int type, bool keep_nyquist, GemmTable* out);
int gemm_kpad(int bins);
// Device bytes of the three-term BF16 row split the tensor-core filter needs.
size_t filter_gemm_split_bytes(int nz, int na, int bins);
// Operand split (three BF16 terms of every row) and the zero guard bins; then
// the tensor-core product itself.
cudaError_t launch_filter_gemm_prep(const float* d_sino, int nz, int na, const PadGeom& g, const FiltLayout& fl,
                                    const GemmTable& tab, float4* d_filt, void* d_split, cudaStream_t st);
cudaError_t launch_filter_gemm(const float* d_sino, int nz, int na, const PadGeom& g, const FiltLayout& fl,
                               const GemmTable& tab, const float4* d_stats, int denorm, float scale,
                               float4* d_filt, void* d_split, unsigned* d_err, cudaStream_t st);

// ---------------------------------------------------------- batched work
// A batch is a table of jobs passed by value as a kernel parameter; a
// persistent grid takes work items from an atomic counter. Each output value
// is produced by exactly one item with a fixed order of operations, so a job's
// result does not depend on what else shares the batch.
constexpr int kMaxJobs = 64;

// Backprojection job: items are (slice group, tile) pairs, slice-group major.
struct BpJob {
    const float4* filt;   // [nzg][na][pitch] float4
    float* out;           // [nz][n][n]
    const float4* stats;  // per-slice {min, max, ...} or null
    Trig trig;
    double ctr;           // voxel-grid centre: floor(n/2) (SerialBackend) or (n-1)/2 (CUDA backend)
    double dc;            // detector centre: floor(sq/2) or (sq-1)/2
    int nz, na, sq, guard, pitch, n, denorm;
    int edge_rule;        // 1: SerialBackend's tap rule (both taps in range); 0: per-tap bounds
    int tiles_x, tiles;   // tiles per row / per slice group
    long long first;      // index of the job's first item in the batch
};
struct BpBatch {
    int njobs = 0;
    long long total = 0;
    BpJob job[kMaxJobs];
};
// Filtering job: items are (slice pair, angle), slice-pair major. All jobs of a
// batch share the convolution length Lc (and so the twiddle table).
struct FiltJob {
    const float* sino;    // [nz][na][bins]
    float4* filt;         // [nzg][na][pitch]
    const float4* stats;
    const float2* Hc;     // convolution spectrum / Lc
    int nz, na, bins, sq, pad, guard, pitch, denorm;  // pad: pad_before, folded into Hc (rows sit at 0)
    float scale;
    long long first;
};
struct FiltBatch {
    int njobs = 0;
    int Lc = 0;
    long long total = 0;
    const float2* tw = nullptr;  // fft_twiddle_table(Lc)
    long long twlen = 0;         // its float2 part (set by launch_filter_batch)
    FiltJob job[kMaxJobs];
};
// Conventions of a reconstruction: SerialBackend's (the default, the oracle)
// or the reference CUDA backend's (CUDABackend.cu).
enum Convention { kConvSerial = 0, kConvCuda = 1 };
BpJob make_bp_job(const float4* d_filt, int nz, int na, const FiltLayout& fl, int n_out, Trig trig,
                  const float4* d_stats, int denorm, float* d_out, int variant, int convention = kConvSerial);
FiltJob make_filt_job(const float* d_sino, int nz, int na, const PadGeom& g, const FiltLayout& fl,
                      const float2* d_Hc, const float4* d_stats, int denorm, float scale,
                      float4* d_filt);
// Backprojection of a batch (below 2^31 items, one tile shape): one CTA per
// item, or with `persistent` a grid of resident CTAs drawing items from
// d_counter (zeroed here on the stream). Filtering takes one CTA per item.
cudaError_t launch_backproject_batch(const BpBatch& b, int variant, unsigned* d_counter, unsigned* d_err,
                                     cudaStream_t st, bool persistent = false);
cudaError_t launch_filter_batch(const FiltBatch& b, cudaStream_t st);
cudaError_t launch_backproject(const float4* d_filt, int nz, int na, const FiltLayout& fl,
                               int n_out, Trig trig, const float4* d_stats, int denorm,
                               float* d_out, unsigned* d_err, cudaStream_t st, int variant = 0,
                               int convention = kConvSerial);
// One CTA whose threads wait, at most `limit_us` microseconds each, on an
// mbarrier that nothing completes; each records a timeout in *d_err (the
// timeout path's self-test).
cudaError_t launch_wait_selftest(unsigned limit_us, unsigned* d_err, cudaStream_t st);
cudaError_t launch_point_count(const float* d_vol, long long total, float thr,
                               unsigned* d_block_counts, int blocks, cudaStream_t st);
cudaError_t launch_point_write(const float* d_vol, int nx, int ny, long long total, float thr,
                               const unsigned long long* d_block_offsets, int blocks,
                               float4* d_points, long long cap, cudaStream_t st);
int point_blocks(long long total);

// Number of kernel launches one launcher issues (for the launch counter).
constexpr int kFilterLaunches = 1;

}  // namespace ctb

// ------------------------------------------------------------------ context
struct ctb_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::recursive_mutex mu;
    std::string last_error;
    uint64_t launches = 0;
    double last_sino_ms = 0.0;
    double last_recon_ms = 0.0;
    double last_phantom_ms = 0.0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // Copy streams and per-slab events of the host-buffer volume pipeline
    // (created on first use).
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    cudaStream_t fbp_stream = nullptr;  // host volume path: slab k's FBP beside slab k+1's forward
    std::vector<cudaEvent_t> slab_ev;

    // Named workspaces, grown on demand and kept until destruction.
    std::map<std::string, ctb::DevBuf> ws;
    // Cached tables: filter spectra per (L, type), twiddles per L.
    std::map<std::pair<int, int>, ctb::DevBuf> filters;
    std::map<int, ctb::DevBuf> twiddles;
    // Filter implementation (ctb_set_filter_mode) and the tensor-core path's
    // Toeplitz tables per (bins, filter).
    int filter_mode = 0;
    int convention = 0;  // CTB_CONVENTION_SERIAL / CTB_CONVENTION_CUDA
    int fwd_bounds = 1;  // forward projector walks only the non-zero bounds
    std::map<std::pair<int, int>, ctb::GemmTable> gemm_tables;
    // Backprojection tile shape: forced (>= 0), or per size bucket from the
    // autotuner, or bp_default_variant.
    int sms = 0;
    int bp_variant = -1;
    bool autotune = false;
    std::map<std::vector<int>, int> tuned;  // {n bucket, angle bucket, slice-group bucket} -> variant
    // Angle tables: uniform angle sets per count; the last explicit list.
    std::map<int, ctb::DevBuf> trig_uniform;
    std::vector<float> user_angles;
    long long user_angles_gen = 0;  // bumps whenever the explicit angle list changes
    // Forward projector plans (angle groups) per (angle set, w, h, nd).
    struct FwdPlanDev {
        ctb::DevBuf groups, order, rec;  // rec: FwdAngleRec per plan slot
        int ngroups = 0, max_strips = 0;
    };
    std::map<std::vector<long long>, FwdPlanDev> fwd_plans;
    std::vector<long long> img_border_geom;  // geometry the image borders were zeroed for
    unsigned* d_err = nullptr;  // device error word for bounded waits
    int fault_slab = -1;        // host-side fault injection in the volume pipeline (tests)

    // Stage profiling: a ring of event sets, one set per volume reconstruction.
    static constexpr int kProfRing = 256;
    // events 0..4 bracket the stages; event 5 marks the start of the filter's
    // main kernel (after the tensor-core path's operand split)
    static constexpr int kProfEvents = 6;
    bool profiling = false;
    std::vector<cudaEvent_t> prof_ev;  // kProfRing * kProfEvents
    long long prof_calls = 0;
};

namespace ctb {
// Get (or grow) a named device workspace of at least `bytes` bytes.
void* workspace(ctb_ctx* ctx, const std::string& name, size_t bytes);
}
