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
// Work decomposition: a work item is a TX x TY voxel tile of four slices (the
// float4 lanes of the filtered rows) of one job. Per angle, the detector window
// that the tile can touch (WIN bins) is staged into shared memory by the
// bulk-copy engine (cp.async.bulk, completion on an mbarrier), CA angles per
// chunk, double-buffered. The tile origin's detector coordinate is evaluated in
// double precision once per angle and split into the window start and a
// fractional offset, so each thread evaluates u in float on small numbers
// (|u_local| < WIN): the interpolation position is ~10x more accurate than the
// reference's float u of magnitude ~sq. Each of the 256 threads accumulates
// VPT voxels x 4 slices in registers; voxels outside the circle load nothing.
// Six shapes are compiled: four tile shapes with 32-angle chunks (32x32 / 4
// per thread, the default; 64x32 / 8; 32x16 / 2; 16x16 / 1) and the 32x32 tile
// with 16- and 64-angle chunks; bp_default_variant picks one of the first four
// from the job's size, the context's autotuner times all six per size bucket.
//
// One kernel serves both shapes of work: a single job with one CTA per item,
// or a batch of jobs (BpBatch) on a persistent grid that takes items from an
// atomic counter. An item's arithmetic depends only on its job and tile shape,
// so a job's output is bit-identical alone and in any mix of the same shape.
#include <algorithm>
#include <cmath>

#include "ctb_internal.h"

namespace ctb {
namespace {

constexpr int NBUF = 2;       // chunk buffers
constexpr int THREADS = 256;
constexpr float kRound = 12582912.0f;   // 1.5 * 2^23: x + kRound rounds x to an integer
constexpr int kRoundBits = 0x4B400000;  // bit pattern of kRound

// A tile shape: TX x TY voxels of four slices, VPT voxels per thread along x
// (spaced XS = TX / VPT apart), CA angles per staged chunk and WIN bins per
// staged window (>= ceil(sqrt((TX-1)^2 + (TY-1)^2)) + 3 plus rounding margin:
// the taps of every tile position lie in [ws, ws + span + 3)). MINB is the
// launch-bounds occupancy target (registers 65536 / (256 MINB)).
template <int TX_, int TY_, int VPT_, int CA_, int WIN_, int MINB_>
struct Shape {
    static constexpr int TX = TX_, TY = TY_, VPT = VPT_, CA = CA_, WIN = WIN_, MINB = MINB_;
    static constexpr int XS = TX / VPT;
    static_assert(XS * TY == THREADS, "256 threads per CTA");
    static_assert(CA <= THREADS, "one thread per staged angle");
    static_assert(WIN <= kBpWindowMax, "window within the filtered-row guard");
};
using V0 = Shape<32, 32, 4, 32, 52, 4>;  // the general-purpose shape
using V1 = Shape<64, 32, 8, 32, 76, 2>;  // wide tiles: half the staging per voxel
using V2 = Shape<32, 16, 2, 32, 40, 4>;  // half-height tiles: twice the CTAs
using V3 = Shape<16, 16, 1, 32, 28, 4>;  // small tiles for small slices
using V4 = Shape<32, 32, 4, 16, 52, 4>;  // the general shape with 16-angle chunks (half the staging buffer)
using V5 = Shape<32, 32, 4, 64, 52, 2>;  // the general shape with 64-angle chunks (half the chunk barriers)

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
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: gives up once `limit_ns` nanoseconds of the GPU's global timer
// have passed since the first unsuccessful poll (2 s in the kernels; a poll may
// itself suspend for a hardware-defined interval, so the bound is on time, with
// 2^22 polls as a second cap), and reports `code` through the device error word.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned* err,
                                                  unsigned long long limit_ns = 2000000000ull,
                                                  unsigned code = 1u) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned it = 0; it < (1u << 22); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) break;
    }
    if (err) atomicOr(err, code);
    return false;
}

// Self-test of the timeout path: one CTA initialises an mbarrier that expects
// one arrival which never comes (no copy or thread arrives on it), and every
// thread waits on it through the same bounded wait the kernels use. Each wait
// gives up after `limit_us` microseconds and records kWaitSelftestCode; the
// kernel then returns normally. Nothing is in flight when it exits.
constexpr unsigned kWaitSelftestCode = 1u << 4;
__global__ void k_wait_selftest(unsigned limit_us, unsigned* err) {
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    mbar_wait_bounded(&bar, 0, err, 1000ull * limit_us, kWaitSelftestCode);
    __syncthreads();
}

// The fields the inner loop reads every angle come first: one 16-byte
// shared-memory broadcast per warp and angle.
struct AngleRec {
    float f0;  // tile-origin u minus window start
    float c, s;
    int edge;      // the window reaches a detector edge: decide taps like the reference
    int ws;        // window start bin (unguarded coordinates)
    float cf, sf;  // the reference's float cos/sin (edge decisions only)
    int pad;
};

template <class C>
struct BpSmem {
    float4 win[NBUF][C::CA][C::WIN];
    AngleRec rec[NBUF][C::CA];
    unsigned long long bar[NBUF];
};

// Backproject one tile (x0, y0) of slice group zg of job J. `chunks` counts
// the chunks this CTA has consumed so far (mbarrier phases continue across
// items). Returns false when a bounded wait gave up (block-uniform).
template <class C>
__device__ __forceinline__ bool bp_tile(BpSmem<C>& S, const BpJob& J, int zg, int x0, int y0, unsigned& chunks,
                                        unsigned* err) {
    constexpr int TX = C::TX, TY = C::TY, VPT = C::VPT, XS = C::XS, CA = C::CA, WIN = C::WIN;
    const int t = threadIdx.x;
    const int lx = t % XS, ly = t / XS;
    const int n = J.n, nz = J.nz, na = J.na, sq = J.sq;
    const double ctr = J.ctr;  // voxel-grid centre (the mask radius too)
    const float radf = static_cast<float>(ctr);

    float add[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int z = 4 * zg + j;
        float a = 0.0f;
        if (J.stats && J.denorm != CTB_DENORM_NONE && z < nz) {
            const float4 st = J.stats[z];
            // CUDABackend.cu:676-681 adds the minimum only when max > min
            a = (J.denorm == CTB_DENORM_CUDA && !(st.y - st.x > 0.0f)) ? 0.0f : st.x;
        }
        add[j] = a;
    }

    // Tiles entirely outside the reconstruction circle hold only the offset.
    {
        const int xe = min(x0 + TX - 1, n - 1), ye = min(y0 + TY - 1, n - 1);
        const double dx = fmax(0.0, fmax(x0 - ctr, ctr - xe));
        const double dy = fmax(0.0, fmax(y0 - ctr, ctr - ye));
        if (dx * dx + dy * dy > ctr * ctr) {
            const int y = y0 + ly;
#pragma unroll
            for (int k = 0; k < VPT; ++k) {
                const int x = x0 + lx + XS * k;
                if (x >= n || y >= n) continue;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int z = 4 * zg + j;
                    if (z < nz) J.out[(static_cast<long long>(z) * n + y) * n + x] = add[j];
                }
            }
            return true;
        }
    }

    const double dcd = J.dc;
    const float dcf = static_cast<float>(J.dc);
    const double ox = static_cast<double>(x0) - ctr, oy = static_cast<double>(y0) - ctr;
    const float4* plane = J.filt + static_cast<long long>(zg) * na * J.pitch;
    const int nch = (na + CA - 1) / CA;

    auto issue = [&](int c, int b) {
        const int a0 = c * CA;
        const int cnt = min(CA, na - a0);
        if (t < cnt) {
            const int a = a0 + t;
            const double2 tc = J.trig.cs[a];
            const float2 tf = J.trig.csf[a];
            const double uo = ox * tc.x - oy * tc.y + dcd;
            const double umin = uo + fmin(0.0, (TX - 1) * tc.x) + fmin(0.0, -(TY - 1) * tc.y);
            const double umax = uo + fmax(0.0, (TX - 1) * tc.x) + fmax(0.0, -(TY - 1) * tc.y);
            const int ws = static_cast<int>(floor(umin)) - 1;
            AngleRec r;
            r.f0 = static_cast<float>(uo - ws);
            r.c = static_cast<float>(tc.x);
            r.s = static_cast<float>(tc.y);
            r.ws = ws;
            r.cf = tf.x;
            r.sf = tf.y;
            // taps near bin 0 or bin sq-1: the reference's float u decides them
            // (the CUDA backend's per-tap bounds need no rule: bins outside
            // [0, sq) are zeros of the guard)
            r.edge = (J.edge_rule && (umin < 2.0 || umax > sq - 3.0)) ? 1 : 0;
            r.pad = 0;
            S.rec[b][t] = r;
            bulk_load(&S.win[b][t][0], plane + static_cast<long long>(a) * J.pitch + J.guard + ws,
                      WIN * sizeof(float4), &S.bar[b]);
        }
        if (t == 0) mbar_expect_tx(&S.bar[b], static_cast<unsigned>(cnt * WIN * sizeof(float4)));
    };

    float4 acc[VPT];
#pragma unroll
    for (int k = 0; k < VPT; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float fx = static_cast<float>(lx), fy = static_cast<float>(ly);
    // positions inside the reconstruction circle (SerialBackend.cpp:220-224);
    // the others are written as the offset only, so their taps are never loaded
    unsigned inside_mask = 0;
    {
        const float yy = static_cast<float>(y0 + ly) - radf;
#pragma unroll
        for (int k = 0; k < VPT; ++k) {
            const float xx = static_cast<float>(x0 + lx + XS * k) - radf;
            if (!(xx * xx + yy * yy > radf * radf)) inside_mask |= 1u << k;
        }
    }

    // all buffers are idle between items: chunk g of this CTA uses buffer g & 1
    issue(0, chunks & 1);
    __syncthreads();
    for (int c = 0; c < nch; ++c) {
        const unsigned g = chunks + c;
        const int b = g & 1;
        if (c + 1 < nch) issue(c + 1, (g + 1) & 1);
        // A failed wait leaves stale window data; the block then stops as a
        // whole at the barrier below (the decision is block-uniform).
        const bool landed = mbar_wait_bounded(&S.bar[b], (g >> 1) & 1, err);
        const int cnt = min(CA, na - c * CA);
        for (int j = 0; j < cnt; ++j) {
            const AngleRec r = S.rec[b][j];
            const float4* w = S.win[b][j];
            const float ub = fmaf(fx, r.c, fmaf(-fy, r.s, r.f0));
            const float c8 = static_cast<float>(XS) * r.c;
            if (!r.edge) {
                // i = floor(u) by rounding u - 1/2 with the kRound addition (no
                // conversion-unit instructions); at an exact tie u = i + 1 the taps
                // shift to (i, i+1) with weights (0, 1), the same value
                const float ubh = ub - 0.5f;
#pragma unroll
                for (int k = 0; k < VPT; ++k) {
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
                for (int k = 0; k < VPT; ++k) {
                    if (!(inside_mask & (1u << k))) continue;
                    const float u = fmaf(static_cast<float>(k), c8, ub);
                    const float fl = floorf(u);
                    const int i = static_cast<int>(fl);
                    const float xs = static_cast<float>(x0 + lx + XS * k) - radf;
                    const float ys = static_cast<float>(y0 + ly) - radf;
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
        if (!__syncthreads_and(landed)) return false;
    }
    chunks += nch;

    const int y = y0 + ly;
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
        const int x = x0 + lx + XS * k;
        if (x >= n || y >= n) continue;
        const bool inside = inside_mask & (1u << k);
        const float v[4] = {acc[k].x, acc[k].y, acc[k].z, acc[k].w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int z = 4 * zg + j;
            if (z < nz) J.out[(static_cast<long long>(z) * n + y) * n + x] = (inside ? v[j] : 0.0f) + add[j];
        }
    }
    return true;
}

// MODE 0: one job, one CTA per item (job 0 indexed statically keeps its fields
// constant-bank operands). MODE 1: many jobs, one CTA per item, the job found
// from blockIdx.x. MODE 2: a persistent grid whose thread 0 draws items from
// *counter.
template <class C, int MODE>
__global__ void __launch_bounds__(THREADS, C::MINB) k_backproject(const __grid_constant__ BpBatch batch,
                                                                  unsigned* __restrict__ counter,
                                                                  unsigned* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    BpSmem<C>& S = *reinterpret_cast<BpSmem<C>*>(smem_raw);
    __shared__ int s_item;
    if (threadIdx.x == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&S.bar[b], 1);
        mbar_fence_init();
    }
    unsigned chunks = 0;
    if constexpr (MODE == 0) {
        __syncthreads();
        const BpJob& J = batch.job[0];
        const int zg = blockIdx.x / J.tiles;
        const int tl = blockIdx.x - zg * J.tiles;
        bp_tile<C>(S, J, zg, (tl % J.tiles_x) * C::TX, (tl / J.tiles_x) * C::TY, chunks, err);
    } else if constexpr (MODE == 1) {
        __syncthreads();
        const int item = blockIdx.x;
        int j = 0;
        while (j + 1 < batch.njobs && batch.job[j + 1].first <= item) ++j;
        const BpJob& J = batch.job[j];
        const int local = item - static_cast<int>(J.first);
        const int zg = local / J.tiles;
        const int tl = local - zg * J.tiles;
        bp_tile<C>(S, J, zg, (tl % J.tiles_x) * C::TX, (tl / J.tiles_x) * C::TY, chunks, err);
    } else {
        for (;;) {
            if (threadIdx.x == 0) s_item = static_cast<int>(atomicAdd(counter, 1u));
            __syncthreads();
            const int item = s_item;  // totals are below 2^31 (checked at launch)
            if (item >= batch.total) break;
            int j = 0;
            while (j + 1 < batch.njobs && batch.job[j + 1].first <= item) ++j;
            const BpJob& J = batch.job[j];
            const int local = item - static_cast<int>(J.first);
            const int zg = local / J.tiles;
            const int tl = local - zg * J.tiles;
            if (!bp_tile<C>(S, J, zg, (tl % J.tiles_x) * C::TX, (tl / J.tiles_x) * C::TY, chunks, err)) break;
            __syncthreads();  // shared state of this item is dead before the next item's staging
        }
    }
}

template <class C>
cudaError_t set_smem() {
    const int bytes = static_cast<int>(sizeof(BpSmem<C>));
    cudaError_t e = cudaFuncSetAttribute(k_backproject<C, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_backproject<C, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_backproject<C, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

template <class C>
cudaError_t launch_one(const BpBatch& b, unsigned* d_err, cudaStream_t st) {
    cudaError_t e = set_smem<C>();
    if (e != cudaSuccess) return e;
    k_backproject<C, 0><<<static_cast<unsigned>(b.total), THREADS, sizeof(BpSmem<C>), st>>>(b, nullptr, d_err);
    return cudaGetLastError();
}

template <class C>
cudaError_t launch_many(const BpBatch& b, bool persistent, unsigned* d_counter, unsigned* d_err, cudaStream_t st) {
    cudaError_t e = set_smem<C>();
    if (e != cudaSuccess) return e;
    if (!persistent) {
        k_backproject<C, 1><<<static_cast<unsigned>(b.total), THREADS, sizeof(BpSmem<C>), st>>>(b, nullptr, d_err);
        return cudaGetLastError();
    }
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_backproject<C, 2>, THREADS, sizeof(BpSmem<C>));
    const long long grid = std::min<long long>(b.total, static_cast<long long>(sms) * (per_sm > 0 ? per_sm : 1));
    e = cudaMemsetAsync(d_counter, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    k_backproject<C, 2><<<static_cast<unsigned>(grid), THREADS, sizeof(BpSmem<C>), st>>>(b, d_counter, d_err);
    return cudaGetLastError();
}

template <class C>
BpShape shape_of() {
    return BpShape{C::TX, C::TY, C::VPT, C::CA, C::WIN};
}

}  // namespace

cudaError_t launch_wait_selftest(unsigned limit_us, unsigned* d_err, cudaStream_t st) {
    k_wait_selftest<<<1, 64, 0, st>>>(limit_us, d_err);
    return cudaGetLastError();
}

BpShape bp_shape(int variant) {
    switch (variant) {
    case 1: return shape_of<V1>();
    case 2: return shape_of<V2>();
    case 3: return shape_of<V3>();
    case 4: return shape_of<V4>();
    case 5: return shape_of<V5>();
    default: return shape_of<V0>();
    }
}

int bp_default_variant(int n_out, int nz, int sms) {
    // Measured on B200 (fbp of random sinograms, shapes forced): the 32x32
    // tile is fastest once its CTAs reach the SM count (n >= 128 at 64
    // slices); below that smaller tiles win by filling more SMs (n = 64,
    // 16 slices: 16x16 0.025 ms, 32x16 0.031 ms, 32x32 0.044 ms). The 64x32
    // tile never won and is left to the autotuner.
    const long long ctas = static_cast<long long>((n_out + 31) / 32) * ((n_out + 31) / 32) * ((nz + 3) / 4);
    if (ctas >= sms) return 0;
    if (4 * ctas >= sms) return 2;
    return 3;
}

FiltLayout filt_layout(int sq, int n_out) {
    // Every position of every tile grid (n rounded up to whole tiles of any
    // shape, at most kBpTileMax) lies within m = max(r, n_pad - 1 - r) of the
    // centre along each axis, so |u - dc| <= m * sqrt(2); windows start one
    // bin below the tile's minimum and span at most kBpWindowMax bins.
    FiltLayout fl;
    fl.sq = sq;
    const int r = n_out / 2;
    const int n_pad = (n_out + kBpTileMax - 1) / kBpTileMax * kBpTileMax;
    const int m = r > n_pad - 1 - r ? r : n_pad - 1 - r;
    const double reach = m * std::sqrt(2.0) + 3.0;
    const double dc = sq / 2;
    const int left = static_cast<int>(std::ceil(reach + 2.0 - dc));
    const int right = static_cast<int>(std::ceil(dc + reach + kBpWindowMax + 2.0 - sq));
    fl.guard = left > 0 ? left : 0;
    fl.pitch = fl.guard + sq + (right > 0 ? right : 0);
    return fl;
}

BpJob make_bp_job(const float4* d_filt, int nz, int na, const FiltLayout& fl, int n_out, Trig trig,
                  const float4* d_stats, int denorm, float* d_out, int variant, int convention) {
    const BpShape sh = bp_shape(variant);
    BpJob J;
    J.filt = d_filt;
    J.out = d_out;
    J.stats = d_stats;
    J.trig = trig;
    J.nz = nz;
    J.na = na;
    J.sq = fl.sq;
    J.guard = fl.guard;
    J.pitch = fl.pitch;
    J.n = n_out;
    J.denorm = denorm;
    if (convention == kConvCuda) {  // CUDABackend.cu:205-224, 672
        J.ctr = 0.5 * (n_out - 1);
        J.dc = 0.5 * (fl.sq - 1);
        J.edge_rule = 0;
    } else {  // SerialBackend.cpp:205-224
        J.ctr = static_cast<double>(n_out / 2);
        J.dc = static_cast<double>(fl.sq / 2);
        J.edge_rule = 1;
    }
    J.tiles_x = (n_out + sh.tx - 1) / sh.tx;
    J.tiles = J.tiles_x * ((n_out + sh.ty - 1) / sh.ty);
    J.first = 0;
    return J;
}

cudaError_t launch_backproject_batch(const BpBatch& b, int variant, unsigned* d_counter, unsigned* d_err,
                                     cudaStream_t st, bool persistent) {
    if (b.total == 0) return cudaSuccess;
    if (b.total > 0x7fffffffLL) return cudaErrorInvalidValue;
    switch (variant) {
    case 1: return launch_many<V1>(b, persistent, d_counter, d_err, st);
    case 2: return launch_many<V2>(b, persistent, d_counter, d_err, st);
    case 3: return launch_many<V3>(b, persistent, d_counter, d_err, st);
    case 4: return launch_many<V4>(b, persistent, d_counter, d_err, st);
    case 5: return launch_many<V5>(b, persistent, d_counter, d_err, st);
    default: return launch_many<V0>(b, persistent, d_counter, d_err, st);
    }
}

cudaError_t launch_backproject(const float4* d_filt, int nz, int na, const FiltLayout& fl,
                               int n_out, Trig trig, const float4* d_stats, int denorm,
                               float* d_out, unsigned* d_err, cudaStream_t st, int variant, int convention) {
    BpBatch b;
    b.njobs = 1;
    b.job[0] = make_bp_job(d_filt, nz, na, fl, n_out, trig, d_stats, denorm, d_out, variant, convention);
    b.total = static_cast<long long>(b.job[0].tiles) * ((nz + 3) / 4);
    if (b.total > 0x7fffffffLL) return cudaErrorInvalidValue;
    switch (variant) {
    case 1: return launch_one<V1>(b, d_err, st);
    case 2: return launch_one<V2>(b, d_err, st);
    case 3: return launch_one<V3>(b, d_err, st);
    case 4: return launch_one<V4>(b, d_err, st);
    case 5: return launch_one<V5>(b, d_err, st);
    default: return launch_one<V0>(b, d_err, st);
    }
}

}  // namespace ctb
