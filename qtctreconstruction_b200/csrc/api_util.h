// api_util.h — helpers shared by the host-side entry points (status
// reporting, workspace access, device tables) of ctb_api.cu, batch.cu and
// server.cu.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <vector>

#include "ctb_internal.h"

namespace ctb {

constexpr int kMaxAngles = 1 << 16;
constexpr int kMaxFft = 8192;

inline ctb_status fail(ctb_ctx* ctx, ctb_status s, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return s;
}

#define CTB_CUDA(ctx, call)                                                                    \
    do {                                                                                       \
        const cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                                 \
            return fail((ctx), e_ == cudaErrorMemoryAllocation ? CTB_ERR_OOM : CTB_ERR_CUDA,   \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define CTB_LAUNCH(ctx, call)       \
    do {                            \
        CTB_CUDA(ctx, (call));      \
        ++(ctx)->launches;          \
    } while (0)

#define CTB_TRY(expr)                 \
    do {                              \
        const ctb_status s_ = (expr); \
        if (s_ != CTB_OK) return s_;  \
    } while (0)

template <typename T>
inline T* ws(ctb_ctx* ctx, const char* name, size_t count) {
    return static_cast<T*>(workspace(ctx, name, count * sizeof(T)));
}

#define CTB_WS(ctx, var, T, name, count)                                                  \
    T* var = ws<T>((ctx), (name), (count));                                               \
    if (!var) return fail((ctx), CTB_ERR_OOM, "device workspace '%s' (%zu bytes) failed", \
                          (name), static_cast<size_t>(count) * sizeof(T))

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Float degrees 180/na * a (SerialBackend.cpp:126-130).
inline std::vector<float> uniform_angles(int na) {
    std::vector<float> a(na);
    const float step = 180.0f / static_cast<float>(na);
    for (int i = 0; i < na; ++i) a[i] = step * static_cast<float>(i);
    return a;
}

struct Guard {
    ctb_ctx* ctx;
    std::lock_guard<std::recursive_mutex> lock;
    explicit Guard(ctb_ctx* c) : ctx(c), lock(c->mu) { cudaSetDevice(c->device); }
};

// Device angle table (double2 cs[na] then float2 csf[na]) filled from host
// degrees; synchronous on the context's stream.
ctb_status fill_trig(ctb_ctx* ctx, const float* angles_deg, int na, void* table);
// Cached uniform table or the context's explicit-list table.
ctb_status trig_table(ctb_ctx* ctx, const float* angles_deg, int na, Trig* out);
// Cached convolution spectrum per (bins, filter) and twiddles per Lc.
ctb_status filter_tables(ctb_ctx* ctx, const PadGeom& g, int type, const float2** d_Hc,
                         const float2** d_tw, bool keep_nyquist = false);
// Reads and clears the device error word (synchronises the context's stream).
ctb_status check_error_word(ctb_ctx* ctx);
// Autotuner bucket of a backprojection job: {ceil(n / 64), ceil(na / 180),
// floor(log2(slice groups))}.
std::vector<int> bp_bucket(int n_out, int nz, int na);
// The tile shape a context uses for a job without timing anything: forced,
// tuned for the job's bucket, or the default.
int bp_variant_for(const ctb_ctx* ctx, int n_out, int nz, int na);

}  // namespace ctb
