// ctb_api.cu — the extern "C" entry points of libctb200.so (include/ctb200.h)
// and the orchestration of the forward / filter / backprojection stages.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "api_util.h"

namespace ctb {
cudaError_t launch_phantom_sum_boxes(const float* d_params, const int* d_boxes, int k, int nx,
                                     int ny, int nz, float* d_vol, cudaStream_t st);
cudaError_t launch_generator3d_boxes(const float* d_ell, const int* d_boxes, int k, int nx,
                                     int ny, int nz, float radius_mm, float* d_vol,
                                     cudaStream_t st);
void phantom_params(uint64_t seed, int count, float* out);
void phantom_boxes(const float* params, int count, int nx, int ny, int nz, int* boxes);
void generator3d_params(float radius, int count, uint32_t seed, const float* tissue, float* ell);
void generator3d_boxes(const float* ell, int count, int nx, int ny, int nz, float radius,
                       int* boxes);
cudaError_t smem_probe(int sms, float* d_out, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1,
                       double* bytes);

void* workspace(ctb_ctx* ctx, const std::string& name, size_t bytes) {
    DevBuf& b = ctx->ws[name];
    if (b.bytes >= bytes && b.ptr) return b.ptr;
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    const size_t want = std::max<size_t>(bytes, 256);
    if (cudaMalloc(&b.ptr, want) != cudaSuccess) {
        cudaGetLastError();
        b.ptr = nullptr;
        return nullptr;
    }
    b.bytes = want;
    return b.ptr;
}
}  // namespace ctb

using namespace ctb;

namespace ctb {

// Fill a device angle table: na double2 (device sincospi) followed by na
// float2 holding the reference's float cos/sin of degToRad(deg)
// (SerialBackend.cpp:92-95, 198-204; Utils.cpp:44-46), computed here on the
// host with the same libm calls.
// A table upload from pageable host memory, complete on return. A plain
// cudaMemcpy from pageable memory may return before its DMA has landed and is
// ordered only against the legacy default stream, while the kernels run on
// non-blocking streams; the copy is therefore queued on the context's stream
// and waited for.
ctb_status upload(ctb_ctx* ctx, void* dst, const void* src, size_t bytes) {
    CTB_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CTB_OK;
}

ctb_status fill_trig(ctb_ctx* ctx, const float* angles_deg, int na, void* table) {
    std::vector<float2> csf(na);
    for (int a = 0; a < na; ++a) {
        const float th = angles_deg[a] * 3.14159265358979323846f / 180.0f;
        csf[a] = make_float2(std::cos(th), std::sin(th));
    }
    float* d_deg = static_cast<float*>(workspace(ctx, "angles_upload", sizeof(float) * na));
    if (!d_deg) return fail(ctx, CTB_ERR_OOM, "angle upload buffer");
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // previous users of the buffers are done
    CTB_TRY(upload(ctx, d_deg, angles_deg, sizeof(float) * na));
    CTB_TRY(upload(ctx, static_cast<double2*>(table) + na, csf.data(), sizeof(float2) * na));
    CTB_LAUNCH(ctx, launch_trig(d_deg, na, static_cast<double2*>(table), ctx->stream));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CTB_OK;
}

// Angle tables on the device. Uniform angles (angles_deg == NULL: 180/na * a
// in float) are cached per count; an explicit angle list is re-uploaded only
// when it differs from the previous one.
ctb_status trig_table(ctb_ctx* ctx, const float* angles_deg, int na, Trig* out) {
    const size_t bytes = (sizeof(double2) + sizeof(float2)) * na;
    void* table = nullptr;
    if (!angles_deg) {
        auto it = ctx->trig_uniform.find(na);
        if (it == ctx->trig_uniform.end()) {
            const std::vector<float> uni = uniform_angles(na);
            DevBuf b;
            CTB_CUDA(ctx, cudaMalloc(&b.ptr, bytes));
            b.bytes = bytes;
            it = ctx->trig_uniform.emplace(na, b).first;
            CTB_TRY(fill_trig(ctx, uni.data(), na, b.ptr));
        }
        table = it->second.ptr;
    } else {
        table = workspace(ctx, "trig_user", bytes);
        if (!table) return fail(ctx, CTB_ERR_OOM, "angle table");
        if (ctx->user_angles.size() != static_cast<size_t>(na) ||
            std::memcmp(ctx->user_angles.data(), angles_deg, sizeof(float) * na) != 0) {
            ctx->user_angles.clear();
            CTB_TRY(fill_trig(ctx, angles_deg, na, table));
            ctx->user_angles.assign(angles_deg, angles_deg + na);
            ++ctx->user_angles_gen;
        }
    }
    out->cs = static_cast<const double2*>(table);
    out->csf = reinterpret_cast<const float2*>(static_cast<const double2*>(table) + na);
    return CTB_OK;
}

// Convolution spectrum (conv_response) per (fft size, filter, bins), and the
// FFT twiddle tables (fft_twiddle_table) per convolution length.
ctb_status filter_tables(ctb_ctx* ctx, const PadGeom& g, int type, const float2** d_Hc,
                         const float2** d_tw, bool keep_nyquist) {
    const int Lc = g.Lc;
    auto key = std::make_pair(g.bins, type + (keep_nyquist ? 16 : 0));
    auto it = ctx->filters.find(key);
    if (it == ctx->filters.end()) {
        const std::vector<float2> Hc = filter_table(g, type, keep_nyquist);
        DevBuf b;
        CTB_CUDA(ctx, cudaMalloc(&b.ptr, sizeof(float2) * Hc.size()));
        b.bytes = sizeof(float2) * Hc.size();
        CTB_TRY(upload(ctx, b.ptr, Hc.data(), b.bytes));
        it = ctx->filters.emplace(key, b).first;
    }
    auto jt = ctx->twiddles.find(Lc);
    if (jt == ctx->twiddles.end()) {
        const std::vector<float2> tw = fft_twiddle_table(Lc);
        DevBuf b;
        CTB_CUDA(ctx, cudaMalloc(&b.ptr, sizeof(float2) * tw.size()));
        b.bytes = sizeof(float2) * tw.size();
        CTB_TRY(upload(ctx, b.ptr, tw.data(), b.bytes));
        jt = ctx->twiddles.emplace(Lc, b).first;
    }
    *d_Hc = static_cast<const float2*>(it->second.ptr);
    *d_tw = static_cast<const float2*>(jt->second.ptr);
    return CTB_OK;
}

std::vector<int> bp_bucket(int n_out, int nz, int na) {
    int zb = 0;
    for (int zg = (nz + 3) / 4; zg > 1; zg >>= 1) ++zb;
    return {(n_out + 63) / 64, (na + 179) / 180, zb};
}

int bp_variant_for(const ctb_ctx* ctx, int n_out, int nz, int na) {
    if (ctx->bp_variant >= 0) return ctx->bp_variant;
    if (ctx->autotune) {
        auto it = ctx->tuned.find(bp_bucket(n_out, nz, na));
        if (it != ctx->tuned.end()) return it->second;
    }
    return bp_default_variant(n_out, nz, ctx->sms);
}

ctb_status check_error_word(ctb_ctx* ctx) {
    unsigned h = 0;
    CTB_CUDA(ctx, cudaMemcpyAsync(&h, ctx->d_err, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h) {
        cudaMemsetAsync(ctx->d_err, 0, sizeof(unsigned), ctx->stream);
        return fail(ctx, CTB_ERR_TIMEOUT, "a bounded device wait gave up (code %u)", h);
    }
    return CTB_OK;
}

}  // namespace ctb

namespace {

// ------------------------------------------------------------ stages
// Record profiling event `k` of the current set (no-op when `ev` is null).
void mark(ctb_ctx* ctx, cudaEvent_t* ev, int k) {
    if (ev) cudaEventRecord(ev[k], ctx->stream);
}

// Angle groups of the forward projector for this geometry (cached; explicit
// angle lists are keyed by their upload generation).
ctb_status forward_plan_dev(ctb_ctx* ctx, const float* angles_deg, int na, int w, int h, int nd,
                            const Trig& trig, const ctb_ctx::FwdPlanDev** out) {
    const std::vector<long long> key = {angles_deg ? ctx->user_angles_gen : -1, na, w, h, nd};
    auto it = ctx->fwd_plans.find(key);
    if (it == ctx->fwd_plans.end()) {
        std::vector<float> uni;
        if (!angles_deg) {
            uni = uniform_angles(na);
            angles_deg = uni.data();
        }
        const FwdPlan plan = forward_plan(angles_deg, na, w, h, nd);
        ctb_ctx::FwdPlanDev d;
        d.ngroups = static_cast<int>(plan.groups.size() / 4);
        d.max_strips = plan.max_strips;
        // frees the plan's buffers on an early exit, before the cache owns them
        struct Pending {
            ctb_ctx::FwdPlanDev* p;
            ~Pending() {
                if (p) {
                    cudaFree(p->groups.ptr);
                    cudaFree(p->order.ptr);
                    cudaFree(p->rec.ptr);
                }
            }
        } pending{&d};
        CTB_CUDA(ctx, cudaMalloc(&d.groups.ptr, sizeof(int) * plan.groups.size()));
        CTB_CUDA(ctx, cudaMalloc(&d.order.ptr, sizeof(int) * plan.order.size()));
        CTB_TRY(upload(ctx, d.groups.ptr, plan.groups.data(), sizeof(int) * plan.groups.size()));
        CTB_TRY(upload(ctx, d.order.ptr, plan.order.data(), sizeof(int) * plan.order.size()));
        CTB_CUDA(ctx, cudaMalloc(&d.rec.ptr, sizeof(FwdAngleRec) * plan.order.size()));
        // the records come from this angle generation's table (the plan's key)
        CTB_LAUNCH(ctx, launch_fwd_angles(static_cast<const int4*>(d.groups.ptr), d.ngroups,
                                          static_cast<const int*>(d.order.ptr), trig,
                                          static_cast<FwdAngleRec*>(d.rec.ptr), ctx->stream));
        it = ctx->fwd_plans.emplace(key, d).first;
        pending.p = nullptr;
    }
    *out = &it->second;
    return CTB_OK;
}

// volume_path selects the CUDA backend's volume detector centre floor(nd/2)
// (CUDABackend.cu:759) instead of its slice centre (nd-1)/2 (:534); the
// Serial convention has floor(nd/2) everywhere.
ctb_status forward_stage(ctb_ctx* ctx, const float* d_vol, int w, int h, int nz, int na, int nd,
                         const float* angles_deg, float* d_sino, float4* d_stats,
                         cudaEvent_t* ev = nullptr, bool volume_path = false) {
    const int nzg = (nz + 3) / 4;
    const size_t elems = fwd_plane_count(nz) * std::max(fwd_plane_elems(h, w), fwd_plane_elems(w, h));
    CTB_WS(ctx, d_img, float4, "img", elems);
    CTB_WS(ctx, d_imgT, float4, "imgT", elems);
    CTB_WS(ctx, d_box, int4, "fbox", 2 * nzg);  // per group: box, then disc
    const int nband = (h + 7) / 8 + (w + 7) / 8;  // per group: row bands, then column bands
    CTB_WS(ctx, d_band, int2, "fband", static_cast<size_t>(nzg) * nband);
    // zero borders: the planes of every group sit at fixed offsets for a
    // given (w, h), and normalisation writes only their interiors, so the
    // buffers' whole capacity is cleared once whenever the buffers or the plane
    // geometry change; any later group count up to the capacity reuses it
    const size_t cap = std::min(ctx->ws["img"].bytes, ctx->ws["imgT"].bytes) / sizeof(float4);
    const std::vector<long long> geom = {reinterpret_cast<long long>(d_img),
                                         reinterpret_cast<long long>(d_imgT), w, h,
                                         static_cast<long long>(cap)};
    if (ctx->img_border_geom != geom) {
        CTB_CUDA(ctx, cudaMemsetAsync(d_img, 0, sizeof(float4) * cap, ctx->stream));
        CTB_CUDA(ctx, cudaMemsetAsync(d_imgT, 0, sizeof(float4) * cap, ctx->stream));
        ctx->img_border_geom = geom;
    }
    Trig trig;
    CTB_TRY(trig_table(ctx, angles_deg, na, &trig));
    // the non-zero bounds (filled by normalisation) or, without them, none
    int4* box = (ctx->convention == kConvCuda || !ctx->fwd_bounds) ? nullptr : d_box;
    int2* band = box ? d_band : nullptr;
    CTB_LAUNCH(ctx, launch_slice_stats(d_vol, static_cast<long long>(w) * h, nz, d_stats, ctx->stream, box,
                                       band, nband));
    if (ctx->convention == kConvCuda) {
        CTB_LAUNCH(ctx, launch_normalize(d_vol, w, h, nz, d_stats, d_img, nullptr, ctx->stream, 0));
        mark(ctx, ev, 1);
        const float det_center = volume_path ? static_cast<float>(nd / 2) : 0.5f * static_cast<float>(nd - 1);
        CTB_LAUNCH(ctx, launch_raymarch(d_img, w, h, nz, na, nd, det_center, trig.cs, d_sino, ctx->stream));
        return CTB_OK;
    }
    CTB_LAUNCH(ctx, launch_normalize(d_vol, w, h, nz, d_stats, d_img, d_imgT, ctx->stream, 1, box, band));
    mark(ctx, ev, 1);
    const ctb_ctx::FwdPlanDev* plan = nullptr;
    CTB_TRY(forward_plan_dev(ctx, angles_deg, na, w, h, nd, trig, &plan));
    CTB_LAUNCH(ctx, launch_forward(d_img, d_imgT, w, h, nz, na, nd,
                                   static_cast<const int4*>(plan->groups.ptr), plan->ngroups, plan->max_strips,
                                   static_cast<const FwdAngleRec*>(plan->rec.ptr), box, band, d_sino,
                                   ctx->stream));
    return CTB_OK;
}

// Grow every workspace forward_stage and fbp_stage use for a volume of
// nz_max slices of n x n (nd bins, n x n output) to its final size, so that a
// pipeline of smaller slabs never reallocates (cudaFree synchronises the whole
// device) between its launches.
ctb_status reserve_volume_workspaces(ctb_ctx* ctx, int n, int nz_max, int na, int nd) {
    const int nzg = (nz_max + 3) / 4;
    const size_t elems = fwd_plane_count(nz_max) * fwd_plane_elems(n, n);
    const int nband = 2 * ((n + 7) / 8);
    CTB_WS(ctx, d_img, float4, "img", elems);
    CTB_WS(ctx, d_imgT, float4, "imgT", elems);
    CTB_WS(ctx, d_box, int4, "fbox", 2 * nzg);
    CTB_WS(ctx, d_band, int2, "fband", static_cast<size_t>(nzg) * nband);
    const PadGeom g = pad_geometry(nd);
    const FiltLayout fl = filt_layout(g.sq, n);
    CTB_WS(ctx, d_filt, float4, "filt", static_cast<size_t>(nzg) * na * fl.pitch);
    if (ctx->filter_mode == CTB_FILTER_MODE_TC_BF16X3) {
        CTB_WS(ctx, d_split, unsigned char, "gemm_split", filter_gemm_split_bytes(nz_max, na, nd));
        (void)d_split;
    }
    (void)d_img; (void)d_imgT; (void)d_box; (void)d_band; (void)d_filt;
    return CTB_OK;
}

// First job of a size bucket with the autotuner on: time every tile shape on
// this job's own filtered rows (two launches each, CUDA events, synchronous),
// keep the fastest for the bucket. The caller then runs the chosen shape, so
// the output is that shape's.
ctb_status tune_backprojection(ctb_ctx* ctx, const float4* d_filt, int nz, int na, const FiltLayout& fl,
                               int n_out, Trig trig, const float4* d_stats, int denorm, float* d_out,
                               int* variant, int bucket_depth) {
    cudaEvent_t e0, e1;
    CTB_CUDA(ctx, cudaEventCreate(&e0));
    CTB_CUDA(ctx, cudaEventCreate(&e1));
    float best = 0.f;
    int best_v = *variant;
    for (int v = 0; v < kBpVariants; ++v) {
        cudaError_t e = launch_backproject(d_filt, nz, na, fl, n_out, trig, d_stats, denorm, d_out, ctx->d_err,
                                           ctx->stream, v, ctx->convention);  // warm-up
        if (e == cudaSuccess) e = cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < 2 && e == cudaSuccess; ++r)
            e = launch_backproject(d_filt, nz, na, fl, n_out, trig, d_stats, denorm, d_out, ctx->d_err,
                                   ctx->stream, v, ctx->convention);
        if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return fail(ctx, CTB_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
        }
        ctx->launches += 3;
        if (v == 0 || ms < best) {
            best = ms;
            best_v = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->tuned[bp_bucket(n_out, bucket_depth, na)] = best_v;
    *variant = best_v;
    return CTB_OK;
}

// shape_depth: the depth the backprojection tile shape is chosen for (a slab
// of a volume uses the whole volume's, so slabs reproduce one pass bit for bit)
ctb_status fbp_stage(ctb_ctx* ctx, const float* d_sino, int nz, int na, int bins,
                     const float* angles_deg, int n_out, int filter, const float4* d_stats,
                     int denorm, float* d_out, cudaEvent_t* ev = nullptr, int shape_depth = 0) {
    const PadGeom g = pad_geometry(bins);
    if (g.Lc > kMaxFft)
        return fail(ctx, CTB_ERR_UNSUPPORTED, "convolution length %d (bins %d) exceeds %d", g.Lc, bins,
                    kMaxFft);
    const FiltLayout fl = filt_layout(g.sq, n_out);
    const int nzg = (nz + 3) / 4;
    CTB_WS(ctx, d_filt, float4, "filt", static_cast<size_t>(nzg) * na * fl.pitch);
    const float2* d_Hc = nullptr;
    const float2* d_tw = nullptr;
    const bool nyq = ctx->convention == kConvCuda;
    CTB_TRY(filter_tables(ctx, g, filter, &d_Hc, &d_tw, nyq));
    Trig trig;
    CTB_TRY(trig_table(ctx, angles_deg, na, &trig));
    // SerialBackend.cpp:246: pi / (2 na) in float
    const float scale = 3.14159265358979323846f / (2.0f * static_cast<float>(na));
    if (ctx->filter_mode == CTB_FILTER_MODE_TC_BF16X3) {
        const auto key = std::make_pair(bins, filter + (nyq ? 16 : 0));
        auto it = ctx->gemm_tables.find(key);
        if (it == ctx->gemm_tables.end()) {
            GemmTable tab;
            CTB_CUDA(ctx, make_gemm_table(g, filter, nyq, &tab));
            it = ctx->gemm_tables.emplace(key, tab).first;
        }
        CTB_WS(ctx, d_split, unsigned char, "gemm_split", filter_gemm_split_bytes(nz, na, bins));
        CTB_LAUNCH(ctx, launch_filter_gemm_prep(d_sino, nz, na, g, fl, it->second, d_filt, d_split, ctx->stream));
        mark(ctx, ev, 5);
        CTB_LAUNCH(ctx, launch_filter_gemm(d_sino, nz, na, g, fl, it->second, d_stats, denorm, scale, d_filt,
                                           d_split, ctx->d_err, ctx->stream));
    } else {
        mark(ctx, ev, 5);
        CTB_LAUNCH(ctx, launch_filter(d_sino, nz, na, g, fl, d_Hc, d_tw, d_stats, denorm, scale, d_filt,
                                      ctx->stream));
    }
    mark(ctx, ev, 3);
    const int zs = shape_depth > 0 ? shape_depth : nz;
    int variant = bp_variant_for(ctx, n_out, zs, na);
    if (ctx->autotune && ctx->bp_variant < 0 && !ctx->tuned.count(bp_bucket(n_out, zs, na)))
        CTB_TRY(tune_backprojection(ctx, d_filt, nz, na, fl, n_out, trig, d_stats, denorm, d_out, &variant, zs));
    CTB_LAUNCH(ctx, launch_backproject(d_filt, nz, na, fl, n_out, trig, d_stats, denorm, d_out,
                                       ctx->d_err, ctx->stream, variant, ctx->convention));
    return CTB_OK;
}

// Slabs of a host-buffer pipeline: {first slice, slices}, whole 8-slice
// groups (the forward projector's groups, and whole 4-slice groups of the
// filter and backprojector, so that a slab-streamed result equals one pass
// over the whole stack bit for bit), about depth/16 slices each. The host->device
// copy of slab k + 1 and the device->host copy of slab k - 1 run on their own
// streams while slab k is computed. The schedule tapers at both ends (a
// quarter slab, three quarters, double slabs, three quarters, a quarter), so
// the copy in before the first slab and the copy out after the last one,
// which nothing overlaps, are short, while the middle launches are large
// enough to keep their tail waves small; each copy in stays shorter than the
// slab computed beside it.
std::vector<int2> plan_slabs(int depth) {
    constexpr int kSlabs = 16;
    std::vector<int2> slabs;
    if (depth <= 16) {
        slabs.push_back(make_int2(0, depth));
        return slabs;
    }
    const int slab = 8 * ((depth + 8 * kSlabs - 1) / (8 * kSlabs));
    const int rem = depth % 8;  // a partial last group goes at the very end
    const int body = depth - rem;
    const int q = slab >= 32 ? 8 * (slab / 32) : 0;  // a quarter slab, whole groups
    std::vector<int> head, tail;
    if (q > 0 && body >= 4 * slab) {
        head = {q, slab - q};
        tail = {slab - q, q};
    }
    int left = body;
    for (int h : head) left -= h;
    for (int h : tail) left -= h;
    int z = 0;
    for (int h : head) { slabs.push_back(make_int2(z, h)); z += h; }
    const int big = head.empty() ? slab : 2 * slab;
    while (left > 0) {
        const int m = std::min(big, left);
        slabs.push_back(make_int2(z, m));
        z += m;
        left -= m;
    }
    for (int h : tail) { slabs.push_back(make_int2(z, h)); z += h; }
    if (rem > 0) {
        if (!slabs.empty() && slabs.back().y + rem <= slab) slabs.back().y += rem;
        else slabs.push_back(make_int2(z, rem));
    }
    return slabs;
}

// Host-buffer FBP of a sinogram stack sinos[depth][na][bins] into
// out[depth][n_out]^2, streamed in slabs (plan_slabs): slab k + 1's sinograms
// copy in on one stream and slab k - 1's slices copy out on another while slab
// k is filtered and backprojected on the context's stream; two buffers each
// way. With denorm != NONE each slice's min/max come from its own sinogram,
// as the interface's default reconstructVolumeFromSinograms takes them
// (BackendFactory.cpp:41-51). The result equals one pass over the whole stack
// bit for bit (whole 8-slice slabs, the tile shape chosen for the whole
// depth). Copies run at full speed only from page-locked host memory; from
// pageable memory the driver stages them. Sets last_recon_ms to the device
// time from the first slab's compute to the last one's.
ctb_status fbp_host_pipeline(ctb_ctx* ctx, const float* sinos, int depth, int na, int bins,
                             const float* angles_deg, int n_out, int filter, int denorm, float* out) {
    const std::vector<int2> slabs = plan_slabs(depth);
    const int nslab = static_cast<int>(slabs.size());
    int slab = 0;
    for (const int2& sl : slabs) slab = std::max(slab, sl.y);
    const size_t row = static_cast<size_t>(na) * bins, img = static_cast<size_t>(n_out) * n_out;
    const PadGeom g = pad_geometry(bins);
    if (g.Lc > kMaxFft)
        return fail(ctx, CTB_ERR_UNSUPPORTED, "convolution length %d (bins %d) exceeds %d", g.Lc, bins, kMaxFft);
    CTB_WS(ctx, d_sino, float, "h_sino", 2 * static_cast<size_t>(slab) * row);
    CTB_WS(ctx, d_out, float, "h_out", 2 * static_cast<size_t>(slab) * img);
    CTB_WS(ctx, d_stats, float4, "h_stats", 2 * static_cast<size_t>(slab));
    {  // the filter stage's workspaces at their final size: nothing reallocates mid-pipeline
        const FiltLayout fl = filt_layout(g.sq, n_out);
        CTB_WS(ctx, d_filt, float4, "filt", static_cast<size_t>((slab + 3) / 4) * na * fl.pitch);
        (void)d_filt;
        if (ctx->filter_mode == CTB_FILTER_MODE_TC_BF16X3) {
            CTB_WS(ctx, d_split, unsigned char, "gemm_split", filter_gemm_split_bytes(slab, na, bins));
            (void)d_split;
        }
    }
    // tables first: building them synchronises the context's stream
    Trig trig;
    CTB_TRY(trig_table(ctx, angles_deg, na, &trig));
    const float2* d_Hc = nullptr;
    const float2* d_tw = nullptr;
    CTB_TRY(filter_tables(ctx, g, filter, &d_Hc, &d_tw, ctx->convention == kConvCuda));
    if (!ctx->copy_in) {
        CTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking));
        CTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking));
    }
    // events: per buffer {sinograms landed, FBP done (sinograms read, slices
    // ready), slices copied out}; then first and last compute marks
    while (ctx->slab_ev.size() < 8) {
        cudaEvent_t e;
        CTB_CUDA(ctx, cudaEventCreate(&e));
        ctx->slab_ev.push_back(e);
    }
    cudaEvent_t* in_done = &ctx->slab_ev[0];
    cudaEvent_t* fbp_done = &ctx->slab_ev[2];
    cudaEvent_t* out_done = &ctx->slab_ev[4];
    cudaEvent_t* mark = &ctx->slab_ev[6];
    cudaStream_t comp = ctx->stream;
    for (int b = 0; b < 2; ++b) {  // buffers start free, after the caller's prior work
        CTB_CUDA(ctx, cudaEventRecord(fbp_done[b], comp));
        CTB_CUDA(ctx, cudaEventRecord(out_done[b], comp));
    }
    // an exit before the end first drains the three streams: no queued copy
    // may still touch the caller's buffers once the call has returned
    struct Drain {
        ctb_ctx* c;
        cudaStream_t comp;
        bool finished = false;
        ~Drain() {
            if (!finished) {
                cudaStreamSynchronize(c->copy_in);
                cudaStreamSynchronize(comp);
                cudaStreamSynchronize(c->copy_out);
            }
        }
    } drain{ctx, comp};
    for (int k = 0; k < nslab; ++k) {
        const int b = k & 1;
        const int z0 = slabs[k].x, nz = slabs[k].y;
        float* sino_b = d_sino + static_cast<size_t>(b) * slab * row;
        float* out_b = d_out + static_cast<size_t>(b) * slab * img;
        float4* stats_b = d_stats + static_cast<size_t>(b) * slab;
        CTB_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_in, fbp_done[b], 0));  // FBP k - 2 read sino_b
        CTB_CUDA(ctx, cudaMemcpyAsync(sino_b, sinos + static_cast<size_t>(z0) * row, sizeof(float) * nz * row,
                                      cudaMemcpyHostToDevice, ctx->copy_in));
        CTB_CUDA(ctx, cudaEventRecord(in_done[b], ctx->copy_in));
        CTB_CUDA(ctx, cudaStreamWaitEvent(comp, in_done[b], 0));
        CTB_CUDA(ctx, cudaStreamWaitEvent(comp, out_done[b], 0));  // slab k - 2 copied out of out_b
        if (k == 0) CTB_CUDA(ctx, cudaEventRecord(mark[0], comp));
        if (denorm != CTB_DENORM_NONE)
            CTB_LAUNCH(ctx, launch_slice_stats(sino_b, static_cast<long long>(row), nz, stats_b, comp));
        CTB_TRY(fbp_stage(ctx, sino_b, nz, na, bins, angles_deg, n_out, filter,
                          denorm != CTB_DENORM_NONE ? stats_b : nullptr, denorm, out_b, nullptr, depth));
        CTB_CUDA(ctx, cudaEventRecord(fbp_done[b], comp));
        CTB_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_out, fbp_done[b], 0));
        CTB_CUDA(ctx, cudaMemcpyAsync(out + static_cast<size_t>(z0) * img, out_b, sizeof(float) * nz * img,
                                      cudaMemcpyDeviceToHost, ctx->copy_out));
        CTB_CUDA(ctx, cudaEventRecord(out_done[b], ctx->copy_out));
    }
    CTB_CUDA(ctx, cudaEventRecord(mark[1], comp));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->copy_out));
    CTB_CUDA(ctx, cudaStreamSynchronize(comp));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->copy_in));
    drain.finished = true;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, mark[0], mark[1]);
    ctx->last_recon_ms = ms;
    return check_error_word(ctx);
}

ctb_status check_common(ctb_ctx* ctx) {
    if (!ctx) return CTB_ERR_INVALID;
    return CTB_OK;
}

}  // namespace

extern "C" {

const char* ctb_status_string(ctb_status s) {
    switch (s) {
    case CTB_OK: return "ok";
    case CTB_ERR_INVALID: return "invalid argument";
    case CTB_ERR_CUDA: return "CUDA error";
    case CTB_ERR_OOM: return "out of device memory";
    case CTB_ERR_UNSUPPORTED: return "unsupported size";
    case CTB_ERR_NO_DEVICE: return "no sm_100 device";
    case CTB_ERR_TIMEOUT: return "device wait timed out";
    case CTB_ERR_CANCELLED: return "cancelled";
    case CTB_ERR_NOT_FOUND: return "not found";
    case CTB_ERR_BUSY: return "busy";
    }
    return "unknown status";
}

ctb_status ctb_create(ctb_ctx** out, int device) {
    if (!out) return CTB_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return CTB_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        cudaGetLastError();
        return CTB_ERR_NO_DEVICE;
    }
    auto* ctx = new ctb_ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_err, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(ctx->d_err, 0, sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return CTB_ERR_CUDA;
    }
    for (auto& e : ctx->ev) cudaEventCreate(&e);
    ctx->stream = ctx->own_stream;
    ctx->sms = prop.multiProcessorCount;
    *out = ctx;
    return CTB_OK;
}

void ctb_destroy(ctb_ctx* ctx) {
    if (!ctx) return;
    {
        std::lock_guard<std::recursive_mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        for (auto& kv : ctx->ws) cudaFree(kv.second.ptr);
        for (auto& kv : ctx->filters) cudaFree(kv.second.ptr);
        for (auto& kv : ctx->twiddles) cudaFree(kv.second.ptr);
        for (auto& kv : ctx->gemm_tables) cudaFree(kv.second.T.ptr);
        for (auto& kv : ctx->trig_uniform) cudaFree(kv.second.ptr);
        for (auto& kv : ctx->fwd_plans) {
            cudaFree(kv.second.groups.ptr);
            cudaFree(kv.second.order.ptr);
            cudaFree(kv.second.rec.ptr);
        }
        for (auto& e : ctx->prof_ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : ctx->ev)
            if (e) cudaEventDestroy(e);
        if (ctx->d_err) cudaFree(ctx->d_err);
        for (auto& e : ctx->slab_ev) cudaEventDestroy(e);
        if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
        if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
        if (ctx->fbp_stream) cudaStreamDestroy(ctx->fbp_stream);
        if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    }
    delete ctx;
}

const char* ctb_last_error(const ctb_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

ctb_status ctb_set_stream(ctb_ctx* ctx, void* stream) {
    if (!ctx) return CTB_ERR_INVALID;
    Guard g(ctx);
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return CTB_OK;
}

ctb_status ctb_synchronize(ctb_ctx* ctx) {
    if (!ctx) return CTB_ERR_INVALID;
    Guard g(ctx);
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return check_error_word(ctx);
}

double ctb_last_sinogram_ms(const ctb_ctx* ctx) { return ctx ? ctx->last_sino_ms : 0.0; }
double ctb_last_reconstruction_ms(const ctb_ctx* ctx) { return ctx ? ctx->last_recon_ms : 0.0; }
double ctb_last_phantom_ms(const ctb_ctx* ctx) { return ctx ? ctx->last_phantom_ms : 0.0; }
uint64_t ctb_launch_count(const ctb_ctx* ctx) { return ctx ? ctx->launches : 0; }

ctb_status ctb_pad_geometry(int bins, int* square_bins, int* pad_before, int* fft_size) {
    if (bins <= 0 || !square_bins || !pad_before || !fft_size) return CTB_ERR_INVALID;
    const PadGeom g = pad_geometry(bins);
    *square_bins = g.sq;
    *pad_before = g.pad;
    *fft_size = g.L;
    return CTB_OK;
}

ctb_status ctb_filter_response(int fft_size, int filter, float* H) {
    if (fft_size < 2 || (fft_size & (fft_size - 1)) || !H) return CTB_ERR_INVALID;
    const auto v = filter_response(fft_size, filter);
    for (size_t i = 0; i < v.size(); ++i) H[i] = static_cast<float>(v[i]);
    return CTB_OK;
}

ctb_status ctb_set_bp_shape(ctb_ctx* ctx, int variant) {
    if (!ctx || variant < -1 || variant >= kBpVariants) return CTB_ERR_INVALID;
    Guard g(ctx);
    ctx->bp_variant = variant;
    return CTB_OK;
}

ctb_status ctb_bp_shape_info(int variant, int* tile_x, int* tile_y, int* voxels_per_thread,
                             int* angles_per_chunk) {
    if (variant < 0 || variant >= kBpVariants) return CTB_ERR_INVALID;
    const BpShape sh = bp_shape(variant);
    if (tile_x) *tile_x = sh.tx;
    if (tile_y) *tile_y = sh.ty;
    if (voxels_per_thread) *voxels_per_thread = sh.vpt;
    if (angles_per_chunk) *angles_per_chunk = sh.ca;
    return CTB_OK;
}

ctb_status ctb_bp_shape_for(ctb_ctx* ctx, int output_size, int depth, int num_angles, int* variant) {
    if (!ctx || !variant || output_size <= 0 || depth <= 0 || num_angles <= 0) return CTB_ERR_INVALID;
    Guard g(ctx);
    *variant = bp_variant_for(ctx, output_size, depth, num_angles);
    return CTB_OK;
}

ctb_status ctb_set_autotune(ctb_ctx* ctx, int enable) {
    if (!ctx) return CTB_ERR_INVALID;
    Guard g(ctx);
    ctx->autotune = enable != 0;
    return CTB_OK;
}

ctb_status ctb_autotune_table(ctb_ctx* ctx, int* entries, int capacity, int* count) {
    if (!ctx || !count || capacity < 0 || (capacity > 0 && !entries)) return CTB_ERR_INVALID;
    Guard g(ctx);
    int k = 0;
    for (const auto& kv : ctx->tuned) {
        if (k < capacity) {
            for (int i = 0; i < 3; ++i) entries[4 * k + i] = kv.first[i];
            entries[4 * k + 3] = kv.second;
        }
        ++k;
    }
    *count = k;
    return CTB_OK;
}

ctb_status ctb_autotune_load(ctb_ctx* ctx, const int* entries, int count) {
    if (!ctx || count < 0 || (count > 0 && !entries)) return CTB_ERR_INVALID;
    for (int k = 0; k < count; ++k)
        if (entries[4 * k + 3] < 0 || entries[4 * k + 3] >= kBpVariants) return CTB_ERR_INVALID;
    Guard g(ctx);
    for (int k = 0; k < count; ++k)
        ctx->tuned[{entries[4 * k], entries[4 * k + 1], entries[4 * k + 2]}] = entries[4 * k + 3];
    return CTB_OK;
}

ctb_status ctb_set_convention(ctb_ctx* ctx, int convention) {
    if (!ctx || (convention != CTB_CONVENTION_SERIAL && convention != CTB_CONVENTION_CUDA)) return CTB_ERR_INVALID;
    Guard g(ctx);
    ctx->convention = convention;
    return CTB_OK;
}

ctb_status ctb_set_forward_bounds(ctb_ctx* ctx, int enable) {
    if (!ctx || (enable != 0 && enable != 1)) return CTB_ERR_INVALID;
    Guard g(ctx);
    ctx->fwd_bounds = enable;
    return CTB_OK;
}

ctb_status ctb_set_filter_mode(ctb_ctx* ctx, int mode) {
    if (!ctx || (mode != CTB_FILTER_MODE_FFT && mode != CTB_FILTER_MODE_TC_BF16X3)) return CTB_ERR_INVALID;
    Guard g(ctx);
    ctx->filter_mode = mode;
    return CTB_OK;
}

ctb_status ctb_set_profiling(ctb_ctx* ctx, int enable) {
    if (!ctx) return CTB_ERR_INVALID;
    Guard g(ctx);
    if (enable && ctx->prof_ev.empty()) {
        ctx->prof_ev.resize(ctb_ctx::kProfRing * ctb_ctx::kProfEvents);
        for (auto& e : ctx->prof_ev) CTB_CUDA(ctx, cudaEventCreate(&e));
    }
    ctx->profiling = enable != 0;
    return CTB_OK;
}

ctb_status ctb_stage_times(ctb_ctx* ctx, int back, double* ms) {
    if (!ctx || !ms || back < 0 || back >= ctb_ctx::kProfRing || back >= ctx->prof_calls ||
        ctx->prof_ev.empty())
        return fail(ctx, CTB_ERR_INVALID, "ctb_stage_times: no such profiled call");
    Guard g(ctx);
    const long long idx = (ctx->prof_calls - 1 - back) % ctb_ctx::kProfRing;
    cudaEvent_t* ev = &ctx->prof_ev[idx * ctb_ctx::kProfEvents];
    CTB_CUDA(ctx, cudaEventSynchronize(ev[4]));
    for (int k = 0; k < 4; ++k) {
        float t = 0.f;
        CTB_CUDA(ctx, cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
        ms[k] = t;
    }
    return CTB_OK;
}

ctb_status ctb_filter_kernel_ms(ctb_ctx* ctx, int back, double* ms) {
    if (!ctx || !ms || back < 0 || back >= ctb_ctx::kProfRing || back >= ctx->prof_calls ||
        ctx->prof_ev.empty())
        return fail(ctx, CTB_ERR_INVALID, "ctb_filter_kernel_ms: no such profiled call");
    Guard g(ctx);
    const long long idx = (ctx->prof_calls - 1 - back) % ctb_ctx::kProfRing;
    cudaEvent_t* ev = &ctx->prof_ev[idx * ctb_ctx::kProfEvents];
    CTB_CUDA(ctx, cudaEventSynchronize(ev[4]));
    float t = 0.f;
    CTB_CUDA(ctx, cudaEventElapsedTime(&t, ev[5], ev[3]));
    *ms = t;
    return CTB_OK;
}

ctb_status ctb_selftest_bounded_wait(ctb_ctx* ctx, unsigned limit_us) {
    if (!ctx || limit_us == 0 || limit_us > 2000000u) return CTB_ERR_INVALID;
    Guard g(ctx);
    CTB_TRY(check_error_word(ctx));  // a stale error word is not this test's
    CTB_LAUNCH(ctx, launch_wait_selftest(limit_us, ctx->d_err, ctx->stream));
    return check_error_word(ctx);
}

ctb_status ctb_set_fault_injection(ctb_ctx* ctx, int slab) {
    if (!ctx || slab < -1) return CTB_ERR_INVALID;
    Guard g(ctx);
    ctx->fault_slab = slab;
    return CTB_OK;
}

ctb_status ctb_probe_smem_bandwidth(ctb_ctx* ctx, double* gbs) {
    if (!ctx || !gbs) return CTB_ERR_INVALID;
    Guard g(ctx);
    int sms = 0;
    CTB_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    CTB_WS(ctx, d_out, float, "probe_out", 4 * sms);
    double bytes = 0.0;
    CTB_LAUNCH(ctx, smem_probe(sms, d_out, ctx->stream, ctx->ev[0], ctx->ev[1], &bytes));
    ++ctx->launches;  // warm-up launch
    CTB_CUDA(ctx, cudaEventSynchronize(ctx->ev[1]));
    float ms = 0.f;
    CTB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    *gbs = bytes / (ms * 1e-3) / 1e9;
    return CTB_OK;
}

// ------------------------------------------------- device-buffer entry points
ctb_status ctb_forward_d(ctb_ctx* ctx, const float* d_vol, int n, int depth, int num_angles,
                         int detector_bins, const float* angles_deg, float* d_sino,
                         float* d_stats) {
    CTB_TRY(check_common(ctx));
    if (!d_vol || !d_sino || !d_stats || n <= 0 || depth <= 0 || num_angles <= 0 ||
        detector_bins <= 0 || num_angles > kMaxAngles)
        return fail(ctx, CTB_ERR_INVALID, "ctb_forward_d: invalid arguments");
    if (!aligned16(d_stats)) return fail(ctx, CTB_ERR_INVALID, "d_stats must be 16-byte aligned");
    Guard g(ctx);
    return forward_stage(ctx, d_vol, n, n, depth, num_angles, detector_bins, angles_deg, d_sino,
                         reinterpret_cast<float4*>(d_stats));
}

ctb_status ctb_fbp_d(ctb_ctx* ctx, const float* d_sino, int depth, int num_angles, int bins,
                     const float* angles_deg, int output_size, int filter, const float* d_stats,
                     int denorm, float* d_out) {
    CTB_TRY(check_common(ctx));
    if (!d_sino || !d_out || depth <= 0 || num_angles <= 0 || bins <= 0 || output_size <= 0 ||
        num_angles > kMaxAngles || denorm < 0 || denorm > CTB_DENORM_CUDA)
        return fail(ctx, CTB_ERR_INVALID, "ctb_fbp_d: invalid arguments");
    if (d_stats && !aligned16(d_stats)) return fail(ctx, CTB_ERR_INVALID, "d_stats must be 16-byte aligned");
    Guard g(ctx);
    return fbp_stage(ctx, d_sino, depth, num_angles, bins, angles_deg, output_size, filter,
                     reinterpret_cast<const float4*>(d_stats), d_stats ? denorm : CTB_DENORM_NONE,
                     d_out);
}

ctb_status ctb_reconstruct_volume_d(ctb_ctx* ctx, const float* d_vol, int n, int depth,
                                    int num_angles, int detector_bins, int filter, float* d_out) {
    CTB_TRY(check_common(ctx));
    if (!d_vol || !d_out || n <= 0 || depth <= 0 || num_angles <= 0 || detector_bins <= 0 ||
        num_angles > kMaxAngles)
        return fail(ctx, CTB_ERR_INVALID, "ctb_reconstruct_volume_d: invalid arguments");
    Guard g(ctx);
    CTB_WS(ctx, d_sino, float, "sino", static_cast<size_t>(depth) * num_angles * detector_bins);
    CTB_WS(ctx, d_stats, float4, "stats", depth);
    cudaEvent_t* pev = nullptr;
    if (ctx->profiling) {
        pev = &ctx->prof_ev[(ctx->prof_calls % ctb_ctx::kProfRing) * ctb_ctx::kProfEvents];
        ++ctx->prof_calls;
    }
    CTB_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    mark(ctx, pev, 0);
    CTB_TRY(forward_stage(ctx, d_vol, n, n, depth, num_angles, detector_bins, nullptr, d_sino, d_stats,
                          pev, true));
    CTB_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    mark(ctx, pev, 2);
    CTB_TRY(fbp_stage(ctx, d_sino, depth, num_angles, detector_bins, nullptr, n, filter, d_stats,
                      ctx->convention == kConvCuda ? CTB_DENORM_CUDA : CTB_DENORM_SERIAL, d_out, pev));
    CTB_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    mark(ctx, pev, 4);
    return CTB_OK;
}

// --------------------------------------------------- host-buffer entry points
ctb_status ctb_compute_sinogram(ctb_ctx* ctx, const float* slice, int width, int height,
                                int num_angles, int detector_bins, float* sino_out,
                                float* angles_deg_out, float* minmax_out) {
    CTB_TRY(check_common(ctx));
    if (!slice || !sino_out || width <= 0 || height <= 0 || num_angles <= 0 ||
        detector_bins <= 0 || num_angles > kMaxAngles)
        return fail(ctx, CTB_ERR_INVALID, "ctb_compute_sinogram: invalid arguments");
    Guard g(ctx);
    const size_t npx = static_cast<size_t>(width) * height;
    const size_t ns = static_cast<size_t>(num_angles) * detector_bins;
    CTB_WS(ctx, d_in, float, "h_in", npx);
    CTB_WS(ctx, d_sino, float, "h_sino", ns);
    CTB_WS(ctx, d_stats, float4, "h_stats", 1);
    CTB_CUDA(ctx, cudaMemcpyAsync(d_in, slice, npx * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CTB_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    CTB_TRY(forward_stage(ctx, d_in, width, height, 1, num_angles, detector_bins, nullptr, d_sino, d_stats));
    CTB_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    CTB_CUDA(ctx, cudaMemcpyAsync(sino_out, d_sino, ns * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    float4 st;
    CTB_CUDA(ctx, cudaMemcpyAsync(&st, d_stats, sizeof st, cudaMemcpyDeviceToHost, ctx->stream));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    ctx->last_sino_ms = ms;
    if (angles_deg_out) {
        const auto a = uniform_angles(num_angles);
        std::memcpy(angles_deg_out, a.data(), sizeof(float) * num_angles);
    }
    if (minmax_out) { minmax_out[0] = st.x; minmax_out[1] = st.y; }
    return check_error_word(ctx);
}

ctb_status ctb_reconstruct_slice(ctb_ctx* ctx, const float* sino, int num_angles,
                                 int detector_bins, const float* angles_deg, int output_size,
                                 int filter, float* out) {
    return ctb_reconstruct_slice_hu(ctx, sino, num_angles, detector_bins, angles_deg, output_size, filter,
                                    0.0f, 0.0f, out);
}

ctb_status ctb_reconstruct_slice_hu(ctb_ctx* ctx, const float* sino, int num_angles, int detector_bins,
                                    const float* angles_deg, int output_size, int filter, float min_hu,
                                    float max_hu, float* out) {
    CTB_TRY(check_common(ctx));
    if (!sino || !out || !angles_deg || num_angles <= 0 || detector_bins <= 0 ||
        output_size <= 0 || num_angles > kMaxAngles)
        return fail(ctx, CTB_ERR_INVALID, "ctb_reconstruct_slice: invalid arguments");
    Guard g(ctx);
    const size_t ns = static_cast<size_t>(num_angles) * detector_bins;
    const size_t no = static_cast<size_t>(output_size) * output_size;
    CTB_WS(ctx, d_sino, float, "h_sino", ns);
    CTB_WS(ctx, d_out, float, "h_out", no);
    CTB_WS(ctx, d_stats, float4, "h_stats", 1);
    CTB_CUDA(ctx, cudaMemcpyAsync(d_sino, sino, ns * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    // the CUDA backend denormalises with the sinogram's HU range (CUDABackend.cu:676-681);
    // SerialBackend::reconstructSlice returns normalised units
    const bool hu = ctx->convention == kConvCuda && max_hu - min_hu > 0.0f;
    if (hu) {
        const float4 st = make_float4(min_hu, max_hu, max_hu - min_hu, max_hu - min_hu);
        CTB_CUDA(ctx, cudaMemcpyAsync(d_stats, &st, sizeof st, cudaMemcpyHostToDevice, ctx->stream));
    }
    CTB_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    CTB_TRY(fbp_stage(ctx, d_sino, 1, num_angles, detector_bins, angles_deg, output_size, filter,
                      hu ? d_stats : nullptr, hu ? CTB_DENORM_CUDA : CTB_DENORM_NONE, d_out));
    CTB_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    CTB_CUDA(ctx, cudaMemcpyAsync(out, d_out, no * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
    ctx->last_recon_ms = ms;
    return check_error_word(ctx);
}

ctb_status ctb_reconstruct_volume(ctb_ctx* ctx, const float* vol, int n, int depth,
                                  int num_angles, int detector_bins, int filter, float* out) {
    CTB_TRY(check_common(ctx));
    if (!vol || !out || n <= 0 || depth <= 0 || num_angles <= 0 || detector_bins <= 0 ||
        num_angles > kMaxAngles)
        return fail(ctx, CTB_ERR_INVALID, "ctb_reconstruct_volume: invalid arguments");
    Guard g(ctx);
    const std::vector<int2> slabs = plan_slabs(depth);
    const int nslab = static_cast<int>(slabs.size());
    int slab = 0;  // the largest slab: buffer sizes
    for (const int2& sl : slabs) slab = std::max(slab, sl.y);
    const size_t per = static_cast<size_t>(slab) * n * n;
    const size_t per_sino = static_cast<size_t>(slab) * num_angles * detector_bins;
    CTB_WS(ctx, d_in, float, "h_in", 2 * per);
    CTB_WS(ctx, d_out, float, "h_out", 2 * per);
    CTB_WS(ctx, d_sino, float, "sino", 2 * per_sino);
    CTB_WS(ctx, d_stats, float4, "stats", 2 * static_cast<size_t>(slab));
    CTB_TRY(reserve_volume_workspaces(ctx, n, slab, num_angles, detector_bins));
    if (!ctx->copy_in) {
        CTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking));
        CTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking));
    }
    if (!ctx->fbp_stream) CTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->fbp_stream, cudaStreamNonBlocking));
    // Two compute streams: the context's stream runs the forward stages, the
    // FBP stream the filter and backprojection, so slab k's FBP overlaps slab
    // k + 1's forward projection (each kernel's arithmetic is unchanged, so
    // the result is still that of one pass). Buffers, two of each, pass
    // between the streams by events: per buffer {input landed, forward done
    // (input read, sinogram ready), FBP done (sinogram read, output ready),
    // output copied}; per slab {start, forward done, end}.
    const size_t need = 8 + 3 * static_cast<size_t>(nslab);
    while (ctx->slab_ev.size() < need) {
        cudaEvent_t e;
        CTB_CUDA(ctx, cudaEventCreate(&e));
        ctx->slab_ev.push_back(e);
    }
    cudaEvent_t* in_done = &ctx->slab_ev[0];
    cudaEvent_t* fwd_done = &ctx->slab_ev[2];
    cudaEvent_t* fbp_done = &ctx->slab_ev[4];
    cudaEvent_t* out_done = &ctx->slab_ev[6];
    cudaEvent_t* t = &ctx->slab_ev[8];
    cudaStream_t fwd_s = ctx->stream, fbp_s = ctx->fbp_stream;
    for (int b = 0; b < 2; ++b) {  // buffers start free, after the caller's prior work
        CTB_CUDA(ctx, cudaEventRecord(fwd_done[b], fwd_s));
        CTB_CUDA(ctx, cudaEventRecord(fbp_done[b], fwd_s));
        CTB_CUDA(ctx, cudaEventRecord(out_done[b], fwd_s));
    }
    // The FBP stages launch on ctx->stream: it points at the FBP stream for
    // them and is restored on every exit. An exit before the loop completes
    // (a failed launch, copy or workspace) first drains all four streams, so
    // that no queued copy still reads `vol` or writes `out`, and no kernel
    // still uses the slab buffers, once the call has returned.
    struct PipelineExit {
        ctb_ctx* c;
        cudaStream_t keep;
        bool finished = false;
        ~PipelineExit() {
            if (!finished) {
                cudaStreamSynchronize(c->copy_in);
                cudaStreamSynchronize(keep);
                cudaStreamSynchronize(c->fbp_stream);
                cudaStreamSynchronize(c->copy_out);
            }
            c->stream = keep;
        }
    } pipeline_exit{ctx, fwd_s};
    for (int k = 0; k < nslab; ++k) {
        const int b = k & 1;
        const int z0 = slabs[k].x, nz = slabs[k].y;
        const size_t off = static_cast<size_t>(z0) * n * n, cnt = static_cast<size_t>(nz) * n * n;
        float* in_b = d_in + b * per;
        float* out_b = d_out + b * per;
        float* sino_b = d_sino + b * per_sino;
        float4* stats_b = d_stats + b * static_cast<size_t>(slab);
        CTB_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_in, fwd_done[b], 0));  // forward k - 2 read in_b
        CTB_CUDA(ctx, cudaMemcpyAsync(in_b, vol + off, cnt * sizeof(float), cudaMemcpyHostToDevice, ctx->copy_in));
        CTB_CUDA(ctx, cudaEventRecord(in_done[b], ctx->copy_in));
        CTB_CUDA(ctx, cudaStreamWaitEvent(fwd_s, in_done[b], 0));
        CTB_CUDA(ctx, cudaStreamWaitEvent(fwd_s, fbp_done[b], 0));  // FBP k - 2 read sino_b, stats_b
        CTB_CUDA(ctx, cudaEventRecord(t[3 * k], fwd_s));
        ctx->stream = fwd_s;
        CTB_TRY(forward_stage(ctx, in_b, n, n, nz, num_angles, detector_bins, nullptr, sino_b, stats_b, nullptr,
                              true));
        CTB_CUDA(ctx, cudaEventRecord(fwd_done[b], fwd_s));
        if (k == ctx->fault_slab)  // test hook: fail with this slab's copy and forward stage queued
            return fail(ctx, CTB_ERR_CUDA, "injected fault after queuing slab %d of %d", k, nslab);
        CTB_CUDA(ctx, cudaEventRecord(t[3 * k + 1], fwd_s));
        CTB_CUDA(ctx, cudaStreamWaitEvent(fbp_s, fwd_done[b], 0));
        CTB_CUDA(ctx, cudaStreamWaitEvent(fbp_s, out_done[b], 0));  // slab k - 2 copied out of out_b
        ctx->stream = fbp_s;
        CTB_TRY(fbp_stage(ctx, sino_b, nz, num_angles, detector_bins, nullptr, n, filter, stats_b,
                          ctx->convention == kConvCuda ? CTB_DENORM_CUDA : CTB_DENORM_SERIAL, out_b, nullptr,
                          depth));
        ctx->stream = fwd_s;
        CTB_CUDA(ctx, cudaEventRecord(fbp_done[b], fbp_s));
        CTB_CUDA(ctx, cudaEventRecord(t[3 * k + 2], fbp_s));
        CTB_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_out, fbp_done[b], 0));
        CTB_CUDA(ctx, cudaMemcpyAsync(out + off, out_b, cnt * sizeof(float), cudaMemcpyDeviceToHost, ctx->copy_out));
        CTB_CUDA(ctx, cudaEventRecord(out_done[b], ctx->copy_out));
    }
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->copy_out));
    CTB_CUDA(ctx, cudaStreamSynchronize(fbp_s));
    CTB_CUDA(ctx, cudaStreamSynchronize(fwd_s));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->copy_in));
    pipeline_exit.finished = true;
    // stage sums (the stages of neighbouring slabs overlap, so these add up
    // to more than the call's wall time)
    double fwd = 0.0, fbp = 0.0;
    for (int k = 0; k < nslab; ++k) {
        float a = 0.f, c = 0.f;
        cudaEventElapsedTime(&a, t[3 * k], t[3 * k + 1]);
        cudaEventElapsedTime(&c, t[3 * k + 1], t[3 * k + 2]);
        fwd += a;
        fbp += c;
    }
    ctx->last_sino_ms = fwd;
    ctx->last_recon_ms = fbp;
    return check_error_word(ctx);
}

ctb_status ctb_reconstruct_from_sinograms(ctb_ctx* ctx, const float* sinos, int depth,
                                          int num_angles, int bins, const float* angles_deg,
                                          int filter, int denorm, float* out) {
    CTB_TRY(check_common(ctx));
    if (!sinos || !out || !angles_deg || depth <= 0 || num_angles <= 0 || bins <= 0 ||
        num_angles > kMaxAngles || denorm < 0 || denorm > CTB_DENORM_CUDA)
        return fail(ctx, CTB_ERR_INVALID, "ctb_reconstruct_from_sinograms: invalid arguments");
    Guard g(ctx);
    ctx->last_sino_ms = 0.0;
    return fbp_host_pipeline(ctx, sinos, depth, num_angles, bins, angles_deg, bins, filter, denorm, out);
}

ctb_status ctb_fbp(ctb_ctx* ctx, const float* sinos, int depth, int num_angles, int bins,
                   const float* angles_deg, int output_size, int filter, float* out) {
    CTB_TRY(check_common(ctx));
    if (!sinos || !out || depth <= 0 || num_angles <= 0 || num_angles > kMaxAngles || bins <= 0 ||
        output_size <= 0 || filter < 0 || filter > CTB_FILTER_BARTLETT)
        return fail(ctx, CTB_ERR_INVALID, "ctb_fbp: invalid arguments");
    Guard g(ctx);
    return fbp_host_pipeline(ctx, sinos, depth, num_angles, bins, angles_deg, output_size, filter,
                             CTB_DENORM_NONE, out);
}

// ------------------------------------------------------------------ phantoms
ctb_status ctb_phantom_params(uint64_t seed, int count, float* params) {
    if (count < 0 || (count > 0 && !params)) return CTB_ERR_INVALID;
    phantom_params(seed, count, params);
    return CTB_OK;
}

ctb_status ctb_phantom_sum_d(ctb_ctx* ctx, const float* params, int count, int nx, int ny,
                             int nz, float* d_vol) {
    CTB_TRY(check_common(ctx));
    if (count < 0 || (count > 0 && !params) || !d_vol || nx <= 0 || ny <= 0 || nz <= 0 || count > 32767)
        return fail(ctx, CTB_ERR_INVALID, "ctb_phantom_sum_d: invalid arguments");
    Guard g(ctx);
    std::vector<int> boxes(6 * static_cast<size_t>(std::max(count, 1)));
    if (count) phantom_boxes(params, count, nx, ny, nz, boxes.data());
    CTB_WS(ctx, d_p, float, "phantom_params", 16 * static_cast<size_t>(std::max(count, 1)));
    CTB_WS(ctx, d_b, int, "phantom_boxes", boxes.size());
    if (count) {
        CTB_CUDA(ctx, cudaMemcpyAsync(d_p, params, sizeof(float) * 16 * count, cudaMemcpyHostToDevice, ctx->stream));
        CTB_CUDA(ctx, cudaMemcpyAsync(d_b, boxes.data(), sizeof(int) * 6 * count, cudaMemcpyHostToDevice, ctx->stream));
    }
    CTB_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    CTB_LAUNCH(ctx, launch_phantom_sum_boxes(d_p, d_b, count, nx, ny, nz, d_vol, ctx->stream));
    CTB_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    // the host vectors must outlive the asynchronous copies
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
    ctx->last_phantom_ms = ms;
    return CTB_OK;
}

ctb_status ctb_phantom_sum(ctb_ctx* ctx, const float* params, int count, int nx, int ny, int nz,
                           float* vol) {
    CTB_TRY(check_common(ctx));
    if (!vol || nx <= 0 || ny <= 0 || nz <= 0) return fail(ctx, CTB_ERR_INVALID, "ctb_phantom_sum: invalid arguments");
    Guard g(ctx);
    const size_t nv = static_cast<size_t>(nx) * ny * nz;
    CTB_WS(ctx, d_vol, float, "h_out", nv);
    CTB_TRY(ctb_phantom_sum_d(ctx, params, count, nx, ny, nz, d_vol));
    CTB_CUDA(ctx, cudaMemcpyAsync(vol, d_vol, nv * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CTB_OK;
}

ctb_status ctb_generator3d(ctb_ctx* ctx, int nx, int ny, int nz, float radius_mm, int count,
                           uint32_t seed, const float* tissue, float* vol) {
    CTB_TRY(check_common(ctx));
    if (!vol || !tissue || nx <= 0 || ny <= 0 || nz <= 0 || count < 0 || count > 32767)
        return fail(ctx, CTB_ERR_INVALID, "ctb_generator3d: invalid arguments");
    Guard g(ctx);
    const int k = std::max(count, 1);
    std::vector<float> ell(7 * static_cast<size_t>(k), 0.0f);
    std::vector<int> boxes(6 * static_cast<size_t>(k), 0);
    if (count) {
        generator3d_params(radius_mm, count, seed, tissue, ell.data());
        generator3d_boxes(ell.data(), count, nx, ny, nz, radius_mm, boxes.data());
    }
    const size_t nv = static_cast<size_t>(nx) * ny * nz;
    CTB_WS(ctx, d_vol, float, "h_out", nv);
    CTB_WS(ctx, d_e, float, "gen_ell", ell.size());
    CTB_WS(ctx, d_b, int, "gen_boxes", boxes.size());
    CTB_CUDA(ctx, cudaMemcpyAsync(d_e, ell.data(), sizeof(float) * ell.size(), cudaMemcpyHostToDevice, ctx->stream));
    CTB_CUDA(ctx, cudaMemcpyAsync(d_b, boxes.data(), sizeof(int) * boxes.size(), cudaMemcpyHostToDevice, ctx->stream));
    CTB_LAUNCH(ctx, launch_generator3d_boxes(d_e, d_b, count, nx, ny, nz, radius_mm, d_vol, ctx->stream));
    CTB_CUDA(ctx, cudaMemcpyAsync(vol, d_vol, nv * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CTB_OK;
}

// --------------------------------------------------------------- point cloud
ctb_status ctb_extract_point_cloud(ctb_ctx* ctx, const float* vol, int nx, int ny, int nz,
                                   float threshold, float* points, int64_t capacity,
                                   int64_t* count) {
    CTB_TRY(check_common(ctx));
    if (!vol || !count || nx <= 0 || ny <= 0 || nz <= 0 || capacity < 0 || (capacity > 0 && !points))
        return fail(ctx, CTB_ERR_INVALID, "ctb_extract_point_cloud: invalid arguments");
    Guard g(ctx);
    const long long total = static_cast<long long>(nx) * ny * nz;
    const int blocks = point_blocks(total);
    CTB_WS(ctx, d_vol, float, "h_in", total);
    CTB_WS(ctx, d_cnt, unsigned, "pc_counts", blocks);
    CTB_WS(ctx, d_off, unsigned long long, "pc_offsets", blocks);
    CTB_CUDA(ctx, cudaMemcpyAsync(d_vol, vol, total * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CTB_LAUNCH(ctx, launch_point_count(d_vol, total, threshold, d_cnt, blocks, ctx->stream));
    std::vector<unsigned> cnt(blocks);
    std::vector<unsigned long long> off(blocks);
    CTB_CUDA(ctx, cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(unsigned) * blocks, cudaMemcpyDeviceToHost, ctx->stream));
    CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unsigned long long run = 0;
    for (int b = 0; b < blocks; ++b) { off[b] = run; run += cnt[b]; }
    *count = static_cast<int64_t>(run);
    const long long keep = std::min<long long>(static_cast<long long>(run), capacity);
    if (keep > 0) {
        CTB_WS(ctx, d_pts, float4, "pc_points", keep);
        CTB_CUDA(ctx, cudaMemcpyAsync(d_off, off.data(), sizeof(unsigned long long) * blocks, cudaMemcpyHostToDevice, ctx->stream));
        CTB_LAUNCH(ctx, launch_point_write(d_vol, nx, ny, total, threshold, d_off, blocks, d_pts, keep, ctx->stream));
        CTB_CUDA(ctx, cudaMemcpyAsync(points, d_pts, sizeof(float4) * keep, cudaMemcpyDeviceToHost, ctx->stream));
        CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return CTB_OK;
}

}  // extern "C"
