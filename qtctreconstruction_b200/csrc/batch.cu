// batch.cu — many FBP jobs of different sizes in a few launches
// (ctb_batch_create / ctb_batch_run / ctb_fbp_batch_d).
//
// The reference reconstructs one volume per call (IReconstructionBackend.h:
// 39-44); a batch takes a list of (sinogram stack, geometry, filter) jobs and
// runs the filter stage of all jobs that share a convolution length in one
// launch and the backprojection of all jobs in one persistent launch whose
// work queue holds (job, slice group, tile) items, the jobs with the most
// angles first so that the cheap items fill the tail. Items never share an
// output value, so each job's result is bit-identical to ctb_fbp_d on that job
// alone. With CTB_BATCH_GRAPH the launches are captured once into a CUDA graph
// and each run replays it.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "api_util.h"

using namespace ctb;

struct ctb_batch {
    ctb_ctx* ctx = nullptr;
    int flags = 0;
    std::vector<ctb_fbp_job> jobs;
    std::vector<FiltBatch> filt;  // one launch each
    std::vector<BpBatch> bp;      // one launch each
    std::vector<int> bp_variant;  // tile shape of each backprojection launch
    void* mem = nullptr;          // angle tables + filtered rows of every job
    size_t bytes = 0;
    unsigned* d_counter = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernel_launches = 0;
    double updates = 0.0;
};

namespace {

constexpr size_t kAlign = 256;
size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

ctb_status check_job(ctb_ctx* ctx, const ctb_fbp_job& j, int i) {
    if (!j.sino || !j.out || j.depth <= 0 || j.num_angles <= 0 || j.num_angles > kMaxAngles ||
        j.bins <= 0 || j.output_size <= 0 || j.filter < 0 || j.filter > CTB_FILTER_BARTLETT)
        return fail(ctx, CTB_ERR_INVALID, "batch job %d: invalid arguments", i);
    const PadGeom g = pad_geometry(j.bins);
    if (g.Lc > kMaxFft)
        return fail(ctx, CTB_ERR_UNSUPPORTED, "batch job %d: convolution length %d exceeds %d", i, g.Lc,
                    kMaxFft);
    return CTB_OK;
}

// Issue the batch's launches on the context's stream.
ctb_status issue(ctb_batch* b) {
    ctb_ctx* ctx = b->ctx;
    for (const FiltBatch& f : b->filt) CTB_LAUNCH(ctx, launch_filter_batch(f, ctx->stream));
    for (size_t i = 0; i < b->bp.size(); ++i) {
        const BpBatch& p = b->bp[i];
        const int v = b->bp_variant[i];
        if (b->flags & CTB_BATCH_PER_JOB) {
            const BpJob& J = p.job[0];
            FiltLayout fl;
            fl.sq = J.sq;
            fl.guard = J.guard;
            fl.pitch = J.pitch;
            CTB_LAUNCH(ctx, launch_backproject(J.filt, J.nz, J.na, fl, J.n, J.trig, nullptr,
                                               CTB_DENORM_NONE, J.out, ctx->d_err, ctx->stream, v));
        } else {
            CTB_LAUNCH(ctx, launch_backproject_batch(p, v, b->d_counter, ctx->d_err, ctx->stream,
                                                     (b->flags & CTB_BATCH_PERSISTENT) != 0));
        }
    }
    return CTB_OK;
}

void release(ctb_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->mem) cudaFree(b->mem);
    b->exec = nullptr;
    b->graph = nullptr;
    b->mem = nullptr;
}

ctb_status build(ctb_batch* b) {
    ctb_ctx* ctx = b->ctx;
    const int n = static_cast<int>(b->jobs.size());
    struct Geo {
        PadGeom g;
        FiltLayout fl;
        size_t trig_off, filt_off;
    };
    std::vector<Geo> geo(n);
    size_t off = align_up(sizeof(unsigned long long));
    for (int i = 0; i < n; ++i) {
        const ctb_fbp_job& j = b->jobs[i];
        Geo& q = geo[i];
        q.g = pad_geometry(j.bins);
        q.fl = filt_layout(q.g.sq, j.output_size);
        q.trig_off = off;
        off += align_up((sizeof(double2) + sizeof(float2)) * static_cast<size_t>(j.num_angles));
        q.filt_off = off;
        off += align_up(sizeof(float4) * static_cast<size_t>((j.depth + 3) / 4) * j.num_angles *
                        q.fl.pitch);
        b->updates += static_cast<double>(j.output_size) * j.output_size * j.depth * j.num_angles;
    }
    b->bytes = off;
    CTB_CUDA(ctx, cudaMalloc(&b->mem, off));
    char* base = static_cast<char*>(b->mem);
    b->d_counter = reinterpret_cast<unsigned*>(base);

    std::vector<FiltJob> fj(n);
    std::vector<BpJob> bj(n);
    std::vector<int> var(n);
    for (int i = 0; i < n; ++i) {
        const ctb_fbp_job& j = b->jobs[i];
        const Geo& q = geo[i];
        void* table = base + q.trig_off;
        if (j.angles_deg) {
            CTB_TRY(fill_trig(ctx, j.angles_deg, j.num_angles, table));
        } else {
            const std::vector<float> uni = uniform_angles(j.num_angles);
            CTB_TRY(fill_trig(ctx, uni.data(), j.num_angles, table));
        }
        Trig trig;
        trig.cs = static_cast<const double2*>(table);
        trig.csf = reinterpret_cast<const float2*>(static_cast<const double2*>(table) + j.num_angles);
        const float2* d_Hc = nullptr;
        const float2* d_tw = nullptr;
        CTB_TRY(filter_tables(ctx, q.g, j.filter, &d_Hc, &d_tw));
        // SerialBackend.cpp:246: pi / (2 na) in float
        const float scale = 3.14159265358979323846f / (2.0f * static_cast<float>(j.num_angles));
        float4* d_filt = reinterpret_cast<float4*>(base + q.filt_off);
        fj[i] = make_filt_job(j.sino, j.depth, j.num_angles, q.g, q.fl, d_Hc, nullptr, CTB_DENORM_NONE,
                              scale, d_filt);
        // the shape fbp_d would use for this job alone (no timing here)
        var[i] = bp_variant_for(ctx, j.output_size, j.depth, j.num_angles);
        bj[i] = make_bp_job(d_filt, j.depth, j.num_angles, q.fl, j.output_size, trig, nullptr,
                            CTB_DENORM_NONE, j.out, var[i]);
    }

    const bool per_job = (b->flags & CTB_BATCH_PER_JOB) != 0;
    const int cap = per_job ? 1 : kMaxJobs;
    // filtering: jobs grouped by convolution length, in input order within a class
    std::vector<int> by_lc(n);
    std::iota(by_lc.begin(), by_lc.end(), 0);
    std::stable_sort(by_lc.begin(), by_lc.end(),
                     [&](int x, int y) { return geo[x].g.Lc < geo[y].g.Lc; });
    for (int k = 0; k < n;) {
        FiltBatch f;
        f.Lc = geo[by_lc[k]].g.Lc;
        const float2* d_Hc = nullptr;
        CTB_TRY(filter_tables(ctx, geo[by_lc[k]].g, b->jobs[by_lc[k]].filter, &d_Hc, &f.tw));
        while (k < n && f.njobs < cap && geo[by_lc[k]].g.Lc == f.Lc) {
            FiltJob J = fj[by_lc[k]];
            J.first = f.total;
            f.total += static_cast<long long>(J.na) * ((J.nz + 1) / 2);
            f.job[f.njobs++] = J;
            ++k;
        }
        b->filt.push_back(f);
    }
    // backprojection: one persistent launch per tile shape, most angles first
    // (the most expensive items lead the queue)
    std::vector<int> by_na(n);
    std::iota(by_na.begin(), by_na.end(), 0);
    std::stable_sort(by_na.begin(), by_na.end(), [&](int x, int y) {
        return var[x] != var[y] ? var[x] < var[y] : b->jobs[x].num_angles > b->jobs[y].num_angles;
    });
    if (per_job) std::iota(by_na.begin(), by_na.end(), 0);
    for (int k = 0; k < n;) {
        BpBatch p;
        const int v = var[by_na[k]];
        while (k < n && p.njobs < cap && var[by_na[k]] == v) {
            BpJob J = bj[by_na[k]];
            J.first = p.total;
            p.total += static_cast<long long>(J.tiles) * ((J.nz + 3) / 4);
            p.job[p.njobs++] = J;
            ++k;
        }
        b->bp.push_back(p);
        b->bp_variant.push_back(v);
    }
    b->kernel_launches = static_cast<int>(b->filt.size() + b->bp.size());

    if (b->flags & CTB_BATCH_GRAPH) {
        CTB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        CTB_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
        const uint64_t before = ctx->launches;
        const ctb_status s = issue(b);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        ctx->launches = before;
        if (s != CTB_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        CTB_CUDA(ctx, e);
        b->graph = g;
        CTB_CUDA(ctx, cudaGraphInstantiate(&b->exec, g, 0));
    }
    return CTB_OK;
}

}  // namespace

extern "C" {

ctb_status ctb_batch_create(ctb_ctx* ctx, const ctb_fbp_job* jobs, int njobs, int flags,
                            ctb_batch** out) {
    if (!ctx || !out) return CTB_ERR_INVALID;
    *out = nullptr;
    if (!jobs || njobs <= 0 || (flags & ~(CTB_BATCH_GRAPH | CTB_BATCH_PER_JOB | CTB_BATCH_PERSISTENT)))
        return fail(ctx, CTB_ERR_INVALID, "ctb_batch_create: invalid arguments");
    for (int i = 0; i < njobs; ++i) CTB_TRY(check_job(ctx, jobs[i], i));
    Guard g(ctx);
    auto* b = new ctb_batch();
    b->ctx = ctx;
    b->flags = flags;
    b->jobs.assign(jobs, jobs + njobs);
    const ctb_status s = build(b);
    if (s != CTB_OK) {
        cudaStreamSynchronize(ctx->stream);
        release(b);
        delete b;
        return s;
    }
    *out = b;
    return CTB_OK;
}

ctb_status ctb_batch_run(ctb_batch* b) {
    if (!b) return CTB_ERR_INVALID;
    ctb_ctx* ctx = b->ctx;
    Guard g(ctx);
    if (b->exec) {
        CTB_CUDA(ctx, cudaGraphLaunch(b->exec, ctx->stream));
        ctx->launches += b->kernel_launches;
        return CTB_OK;
    }
    return issue(b);
}

ctb_status ctb_batch_info(const ctb_batch* b, int* launches, double* updates, size_t* device_bytes) {
    if (!b) return CTB_ERR_INVALID;
    if (launches) *launches = b->kernel_launches;
    if (updates) *updates = b->updates;
    if (device_bytes) *device_bytes = b->bytes;
    return CTB_OK;
}

void ctb_batch_destroy(ctb_batch* b) {
    if (!b) return;
    {
        Guard g(b->ctx);
        cudaStreamSynchronize(b->ctx->stream);
        release(b);
    }
    delete b;
}

ctb_status ctb_fbp_batch_d(ctb_ctx* ctx, const ctb_fbp_job* jobs, int njobs) {
    ctb_batch* b = nullptr;
    CTB_TRY(ctb_batch_create(ctx, jobs, njobs, 0, &b));
    ctb_status s = ctb_batch_run(b);
    if (s == CTB_OK) {
        Guard g(ctx);
        s = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? check_error_word(ctx)
                                                               : fail(ctx, CTB_ERR_CUDA, "batch run failed");
    }
    ctb_batch_destroy(b);
    return s;
}

}  // extern "C"
