// forward_proj.cu — the ray-driven forward projector (the RadonTransform stage
// of the FBP path).
//
// The reference's forward projector (SerialBackend::computeSinogram,
// SerialBackend.cpp:59-136) splats every non-zero pixel onto the two detector
// bins around s = (x-cx)cos + (y-cy)sin + floor(nd/2) with linear weights.
// Here the same linear operator is evaluated as a gather: a thread owns one
// detector bin (a ray) of one angle for four slices and walks the ray through
// the image, collecting the pixels whose splat reaches its bin with the tent
// weight 1 - |s - b| (the identical weights (1-frac, frac) of the splat).
// Sinogram stores are coalesced by detector bin.
//
// A CTA owns FB = 128 consecutive bins, one group of up to GMAX = 4 angles that
// share the walked image axis, and four slices (one float4 plane of the
// normalised image). Thread (x, y) takes bin b0 + x for angle y of the group. The ray family is walked along the image axis it is closest to
// (rows when |cos| >= |sin|, else columns of the transposed copy), so every
// step crosses at most three pixels of the gathered axis. Rows are processed
// in chunks of PCH = 8; per chunk the row segments that any ray of any angle
// of the CTA can touch (FW pixels per row) are staged once into shared memory
// by the bulk-copy engine and read by all angles of the group. The image planes carry
// a zero border (kFwdGuard), so a segment never needs filling. Staging is a
// producer/consumer pipeline: two buffers, each with a "full" mbarrier (bytes
// landed) and an "empty" mbarrier (all warps done), so warps never wait on
// one another at a CTA-wide barrier. The host forms the
// groups so that the segment width provably fits (forward_plan). The crossing
// point q*(b, p) is evaluated in double once per chunk and angle and split
// into an integer and a float fraction; within the chunk each thread steps in
// float on small numbers. The two edge rays (bins 0 and nd-1), where the
// reference's rules are discontinuous, decide which pixels count with the
// reference's own float arithmetic (SerialBackend.cpp:109-120) on a separate,
// warp-uniform path.
#include <cmath>

#include "ctb_internal.h"

namespace ctb {
namespace {

constexpr int FB = kFwdRays;
constexpr int PCH = kFwdRows;
constexpr int FW = kFwdWidth;
constexpr int GMAX = kFwdGroup;
constexpr int AY = GMAX;         // angle lanes per CTA (thread (x, y): ray x, angle y)
constexpr int THREADS = FB * AY;
constexpr int FNB = 3;           // chunk buffers (pipeline depth)
constexpr int MAXCH = 512;       // chunk table capacity (walked extent <= 4096)
constexpr float kRound = 12582912.0f;  // 1.5 * 2^23: x + kRound rounds x to an integer
constexpr int kRoundBits = 0x4B400000;  // bit pattern of kRound

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after 2^22 polls (each poll suspends for a
// hardware-defined interval) and reports through the device error word.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned* err) {
    for (unsigned it = 0; it < (1u << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicOr(err, 2u);
    return false;
}

struct FAngle {
    double q0b0;  // q*(b0, p = 0)
    double inv;   // dq*/db = 1 / kq
    double dq;    // dq*/dp = -kp / kq
    float kqf, R, dqf;
    float cr;      // 0.5 - R: ceil(q - R) = round-to-nearest(q + 0.5 - R) via kRound
    float cf, sf;  // the reference's float cos/sin
    int a;
    int p_lo, p_hi;
    int edge;  // an edge ray (bin 0 or nd-1) of this CTA reaches the image at this angle
};

// The fast path: tent weights of the three pixels around the crossing. With
// u0 = (qa - q*) |kq| in [-1, 0) for the first candidate qa = ceil(q* - R),
// the weights 1 - |s - b| of the candidates qa, qa+1, qa+2 are 1 + u0,
// 1 - |u0 + |kq||, and max(0, 1 - 2|kq| - u0) (the first two are never
// negative, the third candidate is beyond reach when |kq| = 1).
__device__ __forceinline__ void walk_chunk(const float4* __restrict__ sg, const FAngle& f, int t,
                                           int p0, int qs, float4& acc) {
    const double qstar = fma(static_cast<double>(p0), f.dq, fma(static_cast<double>(t), f.inv, f.q0b0));
    const double qfl = floor(qstar);
    const float lq0 = static_cast<float>(static_cast<int>(qfl) - qs) + static_cast<float>(qstar - qfl);
    // Every crossing of every ray of the CTA lies in [3, FW - 6] of the segment
    // unless the chunk meets no ray at all (segment start clamped to the
    // plane); never index outside the segment in that case.
    if (!(lq0 + fminf(0.0f, (PCH - 1) * f.dqf) >= 1.5f && lq0 + fmaxf(0.0f, (PCH - 1) * f.dqf) <= FW - 3.0f))
        return;
    const float akq = fabsf(f.kqf);
    const float c2 = 1.0f - 2.0f * akq;
#pragma unroll
    for (int pp = 0; pp < PCH; ++pp) {
        const float qf = fmaf(static_cast<float>(pp), f.dqf, lq0);
        // first candidate ceil(qf - R), rounded by adding 1.5 * 2^23 (FADD and an
        // integer subtract instead of conversion-unit instructions); a tie moves
        // the three candidates by one pixel at distance exactly R (weight 0)
        const float tr = (qf + f.cr) + kRound;
        const int ia = __float_as_int(tr) - kRoundBits;
        const float u0 = ((tr - kRound) - qf) * akq;
        const float w0 = 1.0f + u0;
        const float w1 = 1.0f - fabsf(u0 + akq);
        const float w2 = fmaxf(0.0f, c2 - u0);
        const float4* row = sg + pp * FW + ia;
        const float4 v0 = row[0], v1 = row[1];
        // the third candidate is loaded only where it carries weight
        const float4 v2 = w2 > 0.0f ? row[2] : make_float4(0.f, 0.f, 0.f, 0.f);
        acc.x = fmaf(w2, v2.x, fmaf(w1, v1.x, fmaf(w0, v0.x, acc.x)));
        acc.y = fmaf(w2, v2.y, fmaf(w1, v1.y, fmaf(w0, v0.y, acc.y)));
        acc.z = fmaf(w2, v2.z, fmaf(w1, v1.z, fmaf(w0, v0.z, acc.z)));
        acc.w = fmaf(w2, v2.w, fmaf(w1, v1.w, fmaf(w0, v0.w, acc.w)));
    }
}

// The edge rays: SerialBackend.cpp:109-120 decides, on its own float s, which
// pixels reach bins 0 and nd-1 (bin 0 only from floor(s) == 0; bin nd-1 from
// floor(s) == nd-2 with weight frac and from floor(s) == nd-1 with weight 1).
__device__ __noinline__ float4 walk_chunk_edge(const float4* __restrict__ sg, const FAngle& f, int t,
                                               int p0, int qs, int b, int nd, bool rows, float cxf,
                                               float cyf, float4 acc) {
    const double qstar = fma(static_cast<double>(p0), f.dq, fma(static_cast<double>(t), f.inv, f.q0b0));
    const double qfl = floor(qstar);
    const float lq0 = static_cast<float>(static_cast<int>(qfl) - qs) + static_cast<float>(qstar - qfl);
    if (!(lq0 + fminf(0.0f, (PCH - 1) * f.dqf) >= 1.5f && lq0 + fmaxf(0.0f, (PCH - 1) * f.dqf) <= FW - 3.0f))
        return acc;
    const bool edge = (b == 0 || b == nd - 1);
    const float dcs = static_cast<float>(nd / 2);
    for (int pp = 0; pp < PCH; ++pp) {
        const float qf = fmaf(static_cast<float>(pp), f.dqf, lq0);
        const float qa = ceilf(qf - f.R);
        const int ia = static_cast<int>(qa);
        const float t0 = (qa - qf) * f.kqf;
        for (int k = 0; k < 3; ++k) {
            const float tt = fmaf(static_cast<float>(k), f.kqf, t0);
            float wgt = fmaxf(0.0f, 1.0f - fabsf(tt));
            if (edge) {
                const int qg = qs + ia + k;
                const int pg = p0 + pp;
                const float xg = static_cast<float>(rows ? qg : pg);
                const float yg = static_cast<float>(rows ? pg : qg);
                const float ss = __fadd_rn(__fadd_rn(__fmul_rn(__fsub_rn(xg, cxf), f.cf),
                                                     __fmul_rn(__fsub_rn(yg, cyf), f.sf)), dcs);
                const int i0 = static_cast<int>(floorf(ss));
                wgt = 0.0f;
                if (i0 >= 0 && i0 < nd - 1) {
                    if (i0 == b) wgt = 1.0f - tt;
                    else if (i0 + 1 == b) wgt = 1.0f + tt;
                } else if (i0 == nd - 1 && b == nd - 1) {
                    wgt = 1.0f;
                }
                wgt = fminf(fmaxf(wgt, 0.0f), 1.0f);
            }
            const float4 v = sg[pp * FW + ia + k];
            acc.x = fmaf(wgt, v.x, acc.x);
            acc.y = fmaf(wgt, v.y, acc.y);
            acc.z = fmaf(wgt, v.z, acc.z);
            acc.w = fmaf(wgt, v.w, acc.w);
        }
    }
    return acc;
}

__global__ void __launch_bounds__(THREADS, 2) k_forward(const float4* __restrict__ img,
                                                        const float4* __restrict__ imgT, int w,
                                                        int h, int nz, int na, int nd, Trig trig,
                                                        const int4* __restrict__ groups,
                                                        const int* __restrict__ order,
                                                        float* __restrict__ sino,
                                                        unsigned* __restrict__ err) {
    extern __shared__ __align__(128) float4 seg[];  // [FNB][PCH][FW] staged segments
    __shared__ __align__(8) unsigned long long full[FNB], empty[FNB];
    __shared__ FAngle fa[GMAX];
    __shared__ int qs_tab[MAXCH];

    const int b0 = blockIdx.x * FB;
    const int b1 = min(b0 + FB, nd);  // exclusive
    const int4 grp = groups[blockIdx.y];
    const int cnt = grp.y;
    const bool rows = grp.z == 0;
    const int g = blockIdx.z;  // slice group (4 slices)
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * FB + tx;
    const int lane = tid & 31;
    const int b = b0 + tx;

    const int np = rows ? h : w;  // walked axis
    const int nq = rows ? w : h;  // gathered axis
    const double cq = rows ? 0.5 * (w - 1) : 0.5 * (h - 1);
    const double cp = rows ? 0.5 * (h - 1) : 0.5 * (w - 1);
    const double dcf = static_cast<double>(nd / 2);

    // p range of a ray family [qa, qb] (crossings at p = 0) within reach of the image
    auto prange = [&](double qa, double qb, double dq, double reach, int& lo, int& hi) {
        lo = 0;
        hi = np - 1;
        if (dq != 0.0) {
            const double pa0 = (-reach - qa) / dq, pb0 = (nq - 1 + reach - qa) / dq;
            const double pa1 = (-reach - qb) / dq, pb1 = (nq - 1 + reach - qb) / dq;
            lo = max(0, static_cast<int>(floor(fmin(fmin(pa0, pb0), fmin(pa1, pb1)))) - 1);
            hi = min(np - 1, static_cast<int>(ceil(fmax(fmax(pa0, pb0), fmax(pa1, pb1)))) + 1);
        } else if (fmax(qa, qb) < -reach || fmin(qa, qb) > nq - 1 + reach) {
            hi = -1;
        }
    };

    if (tid < cnt) {
        const int a = order[grp.x + tid];
        const double2 tc = trig.cs[a];
        const double kq = rows ? tc.x : tc.y;
        const double kp = rows ? tc.y : tc.x;
        // s(q, p) = (q - cq) kq + (p - cp) kp + dcf = b  <=>  q = q0(b) + p dq
        FAngle f;
        f.inv = 1.0 / kq;
        f.dq = -kp * f.inv;
        f.q0b0 = cq + (static_cast<double>(b0) - dcf + cp * kp) * f.inv;
        f.kqf = static_cast<float>(kq);
        f.R = static_cast<float>(fabs(f.inv));
        f.cr = 0.5f - f.R;
        f.dqf = static_cast<float>(f.dq);
        const float2 tf = trig.csf[a];
        f.cf = tf.x;
        f.sf = tf.y;
        f.a = a;
        const double reach = fabs(f.inv) + 2.0;
        prange(f.q0b0, f.q0b0 + (b1 - 1 - b0) * f.inv, f.dq, reach, f.p_lo, f.p_hi);
        f.edge = 0;
        for (int eb : {0, nd - 1}) {
            if (eb < b0 || eb >= b1) continue;
            const double qe = f.q0b0 + (eb - b0) * f.inv;
            int lo, hi;
            prange(qe, qe, f.dq, reach, lo, hi);
            if (hi >= lo) f.edge = 1;
        }
        fa[tid] = f;
    }
    if (tid == 0) {
        for (int i = 0; i < FNB; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], THREADS / 32);
        }
        mbar_fence_init();
    }
    __syncthreads();
    int p_lo = np, p_hi = -1;
    for (int j = 0; j < cnt; ++j) {
        if (fa[j].p_hi >= fa[j].p_lo) {
            p_lo = min(p_lo, fa[j].p_lo);
            p_hi = max(p_hi, fa[j].p_hi);
        }
    }
    const bool live = b < nd;
    const int ja = ty;  // this thread's angle of the group
    const bool has_a = ja < cnt;
    if (p_hi < p_lo) {  // no ray of this CTA meets the image
        if (live)
            for (int k = 0; k < 4; ++k) {
                const int z = 4 * g + k;
                if (z >= nz) break;
                if (has_a) sino[(static_cast<long long>(z) * na + fa[ja].a) * nd + b] = 0.0f;
            }
        return;
    }
    const int nch = (p_hi - p_lo + PCH) / PCH;
    // first staged pixel of every chunk: minimum crossing over angles and corners,
    // kept inside the zero-bordered plane
    for (int ci = tid; ci < nch; ci += THREADS) {
        const double p0 = p_lo + ci * PCH;
        double m = 1e300;
        for (int j = 0; j < cnt; ++j) {
            const double qa0 = fma(p0, fa[j].dq, fa[j].q0b0);
            const double qa1 = qa0 + (b1 - 1 - b0) * fa[j].inv;
            const double e = (PCH - 1) * fa[j].dq;
            m = fmin(m, fmin(fmin(qa0, qa1), fmin(qa0 + e, qa1 + e)));
        }
        const int qs = static_cast<int>(fmax(floor(m), -1e9)) - 3;
        qs_tab[ci] = min(max(qs, -kFwdGuard), nq + kFwdGuard - FW);
    }
    __syncthreads();

    const long long pitch = nq + 2 * kFwdGuard;
    const float4* plane = (rows ? img : imgT) + static_cast<long long>(g) * (np + PCH) * pitch + kFwdGuard;

    // producer (thread 0): stage chunk ci into buffer buf; rows p0..p0+7 exist
    // in the bordered plane, every row copy is FW pixels
    auto issue = [&](int ci, int buf) {
        const int p0 = p_lo + ci * PCH;
        const int qs = qs_tab[ci];
        mbar_expect_tx(&full[buf], PCH * FW * sizeof(float4));
        for (int r = 0; r < PCH; ++r)
            bulk_load(seg + (buf * PCH + r) * FW, plane + static_cast<long long>(p0 + r) * pitch + qs,
                      FW * sizeof(float4), &full[buf]);
    };

    // rows this warp's 32 rays can touch, per angle (warp-uniform): chunks
    // outside them are skipped by the whole warp
    int wlo_a = np, whi_a = -1;
    {
        const int wf = b0 + (tx & ~31), wl = min(wf + 31, nd - 1);
        if (wf < nd && has_a) {
            const FAngle& f = fa[ja];
            prange(f.q0b0 + (wf - b0) * f.inv, f.q0b0 + (wl - b0) * f.inv, f.dq, fabs(f.inv) + 2.0, wlo_a, whi_a);
        }
    }

    // warps holding an edge ray that meets the image take the reference-decision path
    const int wb0 = b0 + (tx & ~31);
    const bool holds_edge = (wb0 <= 0 && 0 < wb0 + 32) || (wb0 <= nd - 1 && nd - 1 < wb0 + 32);
    const bool edge_a = holds_edge && has_a && fa[ja].edge;
    const float cxf = static_cast<float>(w - 1) * 0.5f, cyf = static_cast<float>(h - 1) * 0.5f;

    float4 acc_a = make_float4(0.f, 0.f, 0.f, 0.f);
    int last_issued = -1;  // producer only
    if (tid == 0)
        for (int ci = 0; ci < FNB - 1 && ci < nch; ++ci) {
            issue(ci, ci);
            last_issued = ci;
        }
    bool ok = true;
    for (int ci = 0; ci < nch; ++ci) {
        const int buf = ci % FNB;
        const int nxt = ci + FNB - 1;
        if (tid == 0 && nxt < nch) {
            // the buffer of chunk nxt last held chunk ci-1: wait until all warps released it
            const int nb = nxt % FNB;
            if (ci >= 1 && !mbar_wait_bounded(&empty[nb], ((ci - 1) / FNB) & 1, err)) ok = false;
            if (ok) {
                issue(nxt, nb);
                last_issued = nxt;
            }
        }
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0 && ok;
        if (!ok || !mbar_wait_bounded(&full[buf], (ci / FNB) & 1, err)) { ok = false; break; }
        const int p0 = p_lo + ci * PCH;
        const int qs = qs_tab[ci];
        const float4* sg = seg + buf * PCH * FW;
        if (live) {
            if (has_a && p0 <= whi_a && p0 + PCH - 1 >= wlo_a) {
                if (edge_a) acc_a = walk_chunk_edge(sg, fa[ja], tx, p0, qs, b, nd, rows, cxf, cyf, acc_a);
                else walk_chunk(sg, fa[ja], tx, p0, qs, acc_a);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[buf]);
    }
    if (!ok) {
        // a bounded wait gave up: let the producer's copies in flight land (again
        // bounded) before the CTA's shared memory is released
        if (tid == 0 && last_issued >= 0)
            mbar_wait_bounded(&full[last_issued % FNB], (last_issued / FNB) & 1, nullptr);
        return;
    }
    if (!live) return;
    const float ra[4] = {acc_a.x, acc_a.y, acc_a.z, acc_a.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int z = 4 * g + k;
        if (z >= nz) break;
        if (has_a) sino[(static_cast<long long>(z) * na + fa[ja].a) * nd + b] = ra[k];
    }
}

}  // namespace

cudaError_t launch_forward(const float4* d_img, const float4* d_imgT, int w, int h, int nz,
                           int na, int nd, Trig trig, const int4* d_groups, int ngroups,
                           const int* d_order, float* d_sino, unsigned* d_err, cudaStream_t st) {
    const size_t smem = sizeof(float4) * FNB * PCH * FW;
    const cudaError_t e = cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const int np = w > h ? w : h;
    if ((np + PCH - 1) / PCH + 1 > MAXCH) return cudaErrorInvalidValue;
    const dim3 grid((nd + FB - 1) / FB, ngroups, (nz + 3) / 4);
    k_forward<<<grid, dim3(FB, AY), smem, st>>>(d_img, d_imgT, w, h, nz, na, nd, trig, d_groups,
                                                d_order, d_sino, d_err);
    return cudaGetLastError();
}

}  // namespace ctb
