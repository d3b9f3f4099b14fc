// backproject.cu — pixel-driven backprojection (the BP stage of
// SerialBackend::reconstructSlice, SerialBackend.cpp:197-252).
//
// For a voxel (x, y) of an n x n slice, with r = floor(n/2), xx = x - r,
// yy = y - r and dc = floor(sq/2), the reference sums over angles the linear
// interpolation of the filtered row at u = xx cos - yy sin + dc, taking a
// contribution only when both taps floor(u) and floor(u)+1 lie in [0, sq), and
// zeroes voxels outside the inscribed circle xx^2 + yy^2 > r^2. The result is
// scaled by pi/(2 na) (folded into the filter output here) and, for volume
// reconstruction, denormalised with the slice's span and minimum (span folded
// into the filter output, minimum added in the epilogue).
//
// Work decomposition: a CTA owns a 32 x 32 voxel tile of four slices (the
// float4 lanes of the filtered rows). Per angle, the detector window that the
// tile can touch (kBpWindow bins) is staged into shared memory by the bulk-copy
// engine (cp.async.bulk, completion on an mbarrier), 32 angles per chunk,
// double-buffered. The tile origin's detector coordinate is evaluated in
// double precision once per angle and split into the window start and a
// fractional offset, so each thread evaluates u in float on small numbers
// (|u_local| < 48): the interpolation position is ~10x more accurate than the
// reference's float u of magnitude ~sq. Each thread accumulates 4 voxels x 4
// slices in registers.
#include <cmath>

#include "ctb_internal.h"

namespace ctb {
namespace {

constexpr int TILE = kBpTile;
constexpr int WIN = kBpWindow;
constexpr int CA = 32;        // angles per chunk
constexpr int NBUF = 2;       // chunk buffers
constexpr int THREADS = 256;  // 8 (x) x 32 (y) threads, 4 x-positions each
constexpr float kRound = 12582912.0f;   // 1.5 * 2^23: x + kRound rounds x to an integer
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
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}" :
        "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait: gives up after `limit` polls (each poll itself suspends for a
// hardware-defined interval) and reports through the device error word.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned* err) {
    for (unsigned it = 0; it < (1u << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicOr(err, 1u);
    return false;
}

struct AngleRec {
    float f0;  // tile-origin u minus window start
    float c, s;
    int ws;    // window start bin (unguarded coordinates)
    float cf, sf;  // the reference's float cos/sin (edge decisions only)
    int edge;      // the window reaches a detector edge: decide taps like the reference
    int pad;
};

__global__ void __launch_bounds__(THREADS) k_backproject(
    const float4* __restrict__ filt, int nz, int na, int sq, int guard, int pitch, int n,
    Trig trig, const float4* __restrict__ stats, int denorm, float* __restrict__ out,
    unsigned* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto win = reinterpret_cast<float4 (*)[CA][WIN]>(smem_raw);
    auto rec = reinterpret_cast<AngleRec (*)[CA]>(smem_raw + sizeof(float4) * NBUF * CA * WIN);
    auto bar = reinterpret_cast<unsigned long long*>(smem_raw + sizeof(float4) * NBUF * CA * WIN +
                                                     sizeof(AngleRec) * NBUF * CA);

    const int zg = blockIdx.z;
    const int x0 = blockIdx.x * TILE, y0 = blockIdx.y * TILE;
    const int t = threadIdx.x;
    const int lx = t & 7, ly = t >> 3;
    const int rad = n / 2;
    const float radf = static_cast<float>(rad);

    float add[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int z = 4 * zg + j;
        add[j] = (stats && denorm != CTB_DENORM_NONE && z < nz) ? stats[z].x : 0.0f;
    }

    // Tiles entirely outside the reconstruction circle hold only the offset.
    {
        const int xe = min(x0 + TILE - 1, n - 1), ye = min(y0 + TILE - 1, n - 1);
        const long long dx = max(0, max(x0 - rad, rad - xe));
        const long long dy = max(0, max(y0 - rad, rad - ye));
        if (dx * dx + dy * dy > static_cast<long long>(rad) * rad) {
            const int y = y0 + ly;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int x = x0 + lx + 8 * k;
                if (x >= n || y >= n) continue;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int z = 4 * zg + j;
                    if (z < nz) out[(static_cast<long long>(z) * n + y) * n + x] = add[j];
                }
            }
            return;
        }
    }

    if (t == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&bar[b], 1);
        mbar_fence_init();
    }
    __syncthreads();

    const double dcd = static_cast<double>(sq / 2);
    const float dcf = static_cast<float>(sq / 2);
    const double ox = static_cast<double>(x0 - rad), oy = static_cast<double>(y0 - rad);
    const float4* plane = filt + static_cast<long long>(zg) * na * pitch;
    const int nch = (na + CA - 1) / CA;

    auto issue = [&](int c, int b) {
        const int a0 = c * CA;
        const int cnt = min(CA, na - a0);
        if (t < cnt) {
            const int a = a0 + t;
            const double2 tc = trig.cs[a];
            const float2 tf = trig.csf[a];
            const double uo = ox * tc.x - oy * tc.y + dcd;
            const double umin = uo + fmin(0.0, (TILE - 1) * tc.x) + fmin(0.0, -(TILE - 1) * tc.y);
            const double umax = uo + fmax(0.0, (TILE - 1) * tc.x) + fmax(0.0, -(TILE - 1) * tc.y);
            const int ws = static_cast<int>(floor(umin)) - 1;
            AngleRec r;
            r.f0 = static_cast<float>(uo - ws);
            r.c = static_cast<float>(tc.x);
            r.s = static_cast<float>(tc.y);
            r.ws = ws;
            r.cf = tf.x;
            r.sf = tf.y;
            // taps near bin 0 or bin sq-1: the reference's float u decides them
            r.edge = (umin < 2.0 || umax > sq - 3.0) ? 1 : 0;
            r.pad = 0;
            rec[b][t] = r;
            bulk_load(&win[b][t][0], plane + static_cast<long long>(a) * pitch + guard + ws,
                      WIN * sizeof(float4), &bar[b]);
        }
        if (t == 0) mbar_expect_tx(&bar[b], static_cast<unsigned>(cnt * WIN * sizeof(float4)));
    };

    float4 acc[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float fx = static_cast<float>(lx), fy = static_cast<float>(ly);
    // positions inside the reconstruction circle (SerialBackend.cpp:220-224);
    // the others are written as the offset only, so their taps are never loaded
    unsigned inside_mask = 0;
    {
        const float yy = static_cast<float>(y0 + ly) - radf;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float xx = static_cast<float>(x0 + lx + 8 * k) - radf;
            if (!(xx * xx + yy * yy > radf * radf)) inside_mask |= 1u << k;
        }
    }

    issue(0, 0);
    __syncthreads();
    bool ok_all = true;
    for (int c = 0; c < nch; ++c) {
        const int b = c & 1;
        if (c + 1 < nch) issue(c + 1, (c + 1) & 1);
        // A failed wait leaves stale window data; the block then stops as a
        // whole at the barrier below (the decision is block-uniform).
        const bool landed = mbar_wait_bounded(&bar[b], (c >> 1) & 1, err);
        const int cnt = min(CA, na - c * CA);
        for (int j = 0; j < cnt; ++j) {
            const AngleRec r = rec[b][j];
            const float4* w = win[b][j];
            const float ub = fmaf(fx, r.c, fmaf(-fy, r.s, r.f0));
            const float c8 = 8.0f * r.c;
            if (!r.edge) {
                // i = floor(u) by rounding u - 1/2 with the kRound addition (no
                // conversion-unit instructions); at an exact tie u = i + 1 the taps
                // shift to (i, i+1) with weights (0, 1), the same value
                const float ubh = ub - 0.5f;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (!(inside_mask & (1u << k))) continue;
                    const float uh = fmaf(static_cast<float>(k), c8, ubh);
                    const float tr = uh + kRound;
                    const int i = __float_as_int(tr) - kRoundBits;
                    const float d = uh - (tr - kRound);  // frac(u) - 1/2
                    const float w1 = d + 0.5f;
                    const float w0 = 0.5f - d;
                    const float4 lo = w[i], hi = w[i + 1];
                    acc[k].x = fmaf(w1, hi.x, fmaf(w0, lo.x, acc[k].x));
                    acc[k].y = fmaf(w1, hi.y, fmaf(w0, lo.y, acc[k].y));
                    acc[k].z = fmaf(w1, hi.z, fmaf(w0, lo.z, acc[k].z));
                    acc[k].w = fmaf(w1, hi.w, fmaf(w0, lo.w, acc[k].w));
                }
            } else {
                // SerialBackend.cpp:229-239 evaluates u = (xx cos - yy sin) + dc in
                // float without fused multiply-add and keeps the tap pair only when
                // 0 <= floor(u) and floor(u) + 1 < sq; that decision is reproduced
                // here exactly, the interpolation itself uses the accurate u.
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (!(inside_mask & (1u << k))) continue;
                    const float u = fmaf(static_cast<float>(k), c8, ub);
                    const float fl = floorf(u);
                    const int i = static_cast<int>(fl);
                    const float xs = static_cast<float>(x0 + lx + 8 * k - rad);
                    const float ys = static_cast<float>(y0 + ly - rad);
                    const float us = __fadd_rn(__fsub_rn(__fmul_rn(xs, r.cf), __fmul_rn(ys, r.sf)), dcf);
                    const int is = static_cast<int>(floorf(us));
                    const bool ok = (is >= 0) && (is + 1 < sq);
                    const float w1 = ok ? u - fl : 0.0f;
                    const float w0 = ok ? 1.0f - (u - fl) : 0.0f;
                    const float4 lo = w[i], hi = w[i + 1];
                    acc[k].x = fmaf(w1, hi.x, fmaf(w0, lo.x, acc[k].x));
                    acc[k].y = fmaf(w1, hi.y, fmaf(w0, lo.y, acc[k].y));
                    acc[k].z = fmaf(w1, hi.z, fmaf(w0, lo.z, acc[k].z));
                    acc[k].w = fmaf(w1, hi.w, fmaf(w0, lo.w, acc[k].w));
                }
            }
        }
        if (!__syncthreads_and(landed)) { ok_all = false; break; }
    }
    if (!ok_all) return;

    const int y = y0 + ly;
    const float yy = static_cast<float>(y) - radf;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int x = x0 + lx + 8 * k;
        if (x >= n || y >= n) continue;
        const float xx = static_cast<float>(x) - radf;
        const bool inside = !(xx * xx + yy * yy > radf * radf);
        const float v[4] = {acc[k].x, acc[k].y, acc[k].z, acc[k].w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int z = 4 * zg + j;
            if (z < nz) out[(static_cast<long long>(z) * n + y) * n + x] = (inside ? v[j] : 0.0f) + add[j];
        }
    }
}

}  // namespace

FiltLayout filt_layout(int sq, int n_out) {
    // Every position of the tile grid (n rounded up to whole tiles) lies within
    // m = max(r, n_pad - 1 - r) of the centre along each axis, so |u - dc| <=
    // m * sqrt(2); windows start one bin below the tile's minimum and span
    // kBpWindow bins.
    FiltLayout fl;
    fl.sq = sq;
    const int r = n_out / 2;
    const int n_pad = (n_out + kBpTile - 1) / kBpTile * kBpTile;
    const int m = r > n_pad - 1 - r ? r : n_pad - 1 - r;
    const double reach = m * std::sqrt(2.0) + 3.0;
    const double dc = sq / 2;
    const int left = static_cast<int>(std::ceil(reach + 2.0 - dc));
    const int right = static_cast<int>(std::ceil(dc + reach + kBpWindow + 2.0 - sq));
    fl.guard = left > 0 ? left : 0;
    fl.pitch = fl.guard + sq + (right > 0 ? right : 0);
    return fl;
}

cudaError_t launch_backproject(const float4* d_filt, int nz, int na, const FiltLayout& fl,
                               int n_out, Trig trig, const float4* d_stats, int denorm,
                               float* d_out, unsigned* d_err, cudaStream_t st) {
    const dim3 grid((n_out + TILE - 1) / TILE, (n_out + TILE - 1) / TILE, (nz + 3) / 4);
    const size_t smem = sizeof(float4) * NBUF * CA * WIN + sizeof(AngleRec) * NBUF * CA +
                        sizeof(unsigned long long) * NBUF;
    const cudaError_t e = cudaFuncSetAttribute(
        k_backproject, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    k_backproject<<<grid, THREADS, smem, st>>>(d_filt, nz, na, fl.sq, fl.guard, fl.pitch, n_out, trig,
                                               d_stats, denorm, d_out, d_err);
    return cudaGetLastError();
}

}  // namespace ctb
