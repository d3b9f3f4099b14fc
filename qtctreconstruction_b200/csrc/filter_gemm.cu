// filter_gemm.cu — the ramp filter as a dense Toeplitz-matrix product on the
// tcgen05 tensor cores with three-term BF16 splitting (the precision option
// of the filter stage, SerialBackend.cpp:150-195; the FFT path in filter.cu
// stays the default).
//
// Filtered bin i of a sinogram row x is y[i] = sum_j h(i - pad - j) x[j] with
// the lag-domain kernel h of conv_kernel (the same linear operator the FFT
// path applies). Over all rows this is Y[rows x sq] = X[rows x nd] T^T with the
// Toeplitz matrix T[i][j] = h(i - pad - j). Both factors are split into three
// BF16 terms, X = X0 + X1 + X2 and T = T0 + T1 + T2 (each term the BF16
// rounding of what the previous ones leave, about 24 significant bits in
// all), and the six products Xa Tb with a + b <= 2 are accumulated in FP32 in
// tensor memory, smallest first (the dropped terms are about 2^-24 relative).
// Two-term splitting, 16 bits, is not enough: the ramp filter's cancellation
// amplifies its error to ~1e-4 rel-L2 of the reconstruction.
//
// Kernel shape: one CTA per 128-row x BN-bin output tile (BN <= 160, a multiple
// of 16 chosen so that ceil(sq / 160) tiles cover sq with the least waste),
// 128 threads. Thread 0 stages 64-wide K slices of the six operand terms with
// TMA (cp.async.bulk.tensor, 128-byte swizzle, no multicast) into a two-stage ring;
// thread 32 issues tcgen05.mma (kind::f16, BF16 in, FP32 accumulate, M = 128,
// N = BN, K = 16) from shared-memory descriptors and releases each stage with
// tcgen05.commit; after the last slice all four warps read the accumulator
// with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31), scale it, and write
// the filtered rows through shared memory as coalesced float4 runs of the
// backprojector's slice-interleaved layout. Rows of X are ordered
// (slice group, angle, slice % 4) so that four consecutive rows form one
// float4 of the output. Every mbarrier wait is bounded and reports through
// the device error word.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "ctb_internal.h"

namespace ctb {
namespace {

constexpr int BM = 128;
constexpr int BK = 64;          // bf16 per 128-byte swizzle row
constexpr int BNMAX = 160;
constexpr int STAGES = 2;
constexpr int NTERMS = 3;                // BF16 terms per factor
constexpr int A_BYTES = BM * BK * 2;     // 16 KB
constexpr int B_BYTES = BNMAX * BK * 2;  // 20 KB
constexpr int STAGE_BYTES = NTERMS * A_BYTES + NTERMS * B_BYTES;  // 108 KB: two stages fit
static_assert(A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "operand tiles on the 1024-byte swizzle atom");
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + 1024-byte alignment slack
constexpr int TMEM_COLS = 256;
constexpr unsigned kWaitLimit = 1u << 22;

struct GemmParams {
    float4* filt;
    const float4* stats;
    int nz, na, sq, guard, pitch, denorm;
    float scale;
    int bn, nk;
    int pairs;  // nzg * na: output rows of float4
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
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
// Bounded wait: gives up after 2 s of the GPU's global timer from the first
// unsuccessful poll (a poll may itself suspend for a hardware-defined
// interval), or kWaitLimit polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    if (mbar_try_wait(bar, parity)) return true;
    unsigned long long t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (unsigned it = 0; it < kWaitLimit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > 2000000000ull) break;
    }
    return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}
// Shared-memory matrix descriptor of a K-major operand in the 128-byte swizzle
// layout TMA writes: rows of 128 bytes, groups of 8 rows 1024 bytes apart
// (stride byte offset), descriptor version 1, layout type 2 (128-byte swizzle).
__device__ __forceinline__ unsigned long long smem_desc(const void* p) {
    const unsigned long long a = smem_u32(p);
    return ((a >> 4) & 0x3FFFull) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void mma_bf16(unsigned tmem, unsigned long long da, unsigned long long db,
                                         unsigned idesc, unsigned accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_ld16(unsigned addr, float (&v)[16]) {
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Per-slice output scale: pi/(2 na) times the denormalisation span (the FFT
// path's slice_scale).
__device__ __forceinline__ float row_scale(const float4* stats, int z, int nz, int denorm, float scale) {
    if (z >= nz) return 0.0f;
    if (!stats || denorm == CTB_DENORM_NONE) return scale;
    const float4 st = stats[z];
    const float span = st.y - st.x;
    if (denorm == CTB_DENORM_SERIAL) return scale * (span <= 0.0f ? 1.0f : span);
    if (denorm == CTB_DENORM_CUDA) return span > 0.0f ? scale * span : scale;
    return span > 0.0f ? scale * span : 0.0f;
}

// The tensor maps of the six operand terms (X0, X1, X2, T0, T1, T2).
struct GemmMaps {
    CUtensorMap x[NTERMS], t[NTERMS];
};

__global__ void __launch_bounds__(128, 1) k_filter_gemm(const __grid_constant__ GemmMaps maps,
                                                        const GemmParams P, unsigned* __restrict__ err) {
    extern __shared__ unsigned char smem_raw[];
    // 1024-byte alignment of the shared-window offset (the swizzle atom)
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    __shared__ __align__(8) unsigned long long full[STAGES], empty[STAGES], done;
    __shared__ unsigned tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = blockIdx.x * P.bn;
    const int m0 = blockIdx.y * BM;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 32) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_slot;
    const unsigned tx_bytes = NTERMS * A_BYTES + NTERMS * static_cast<unsigned>(P.bn) * BK * 2u;

    if (threadIdx.x == 0) {
        // producer: K slice kt into stage kt % STAGES once the MMAs of slice
        // kt - STAGES have released it
        int issued = 0;
        for (int kt = 0; kt < P.nk; ++kt) {
            const int s = kt % STAGES;
            if (kt >= STAGES && !mbar_wait(&empty[s], ((kt - STAGES) / STAGES) & 1)) {
                atomicOr(err, 4u);
                break;
            }
            unsigned char* st = smem + s * STAGE_BYTES;
            mbar_expect_tx(&full[s], tx_bytes);
#pragma unroll
            for (int a = 0; a < NTERMS; ++a) tma_load_2d(st + a * A_BYTES, &maps.x[a], kt * BK, m0, &full[s]);
#pragma unroll
            for (int b = 0; b < NTERMS; ++b)
                tma_load_2d(st + NTERMS * A_BYTES + b * B_BYTES, &maps.t[b], kt * BK, n0, &full[s]);
            issued = kt + 1;
        }
        if (issued < P.nk) {
            // gave up: let the copies in flight land (bounded) before the CTA ends
            for (int kt = issued > STAGES ? issued - STAGES : 0; kt < issued; ++kt)
                mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1);
        }
    } else if (threadIdx.x == 32) {
        // MMA issuer: 6 products x 4 K steps of 16 per slice, the products of
        // the smaller terms first (a + b = 2, then 1, then 0)
        const unsigned idesc = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<unsigned>(P.bn >> 3) << 17) |
                               (static_cast<unsigned>(BM >> 4) << 24);
        for (int kt = 0; kt < P.nk; ++kt) {
            const int s = kt % STAGES;
            if (!mbar_wait(&full[s], (kt / STAGES) & 1)) {
                atomicOr(err, 8u);
                break;
            }
            tc_fence_after();
            const unsigned char* st = smem + s * STAGE_BYTES;
            constexpr int PA[6] = {2, 1, 0, 1, 0, 0}, PB[6] = {0, 1, 2, 0, 1, 0};
#pragma unroll
            for (int p = 0; p < 6; ++p) {
                const unsigned char* a = st + PA[p] * A_BYTES;
                const unsigned char* b = st + NTERMS * A_BYTES + PB[p] * B_BYTES;
#pragma unroll
                for (int ks = 0; ks < BK / 16; ++ks)
                    mma_bf16(tmem, smem_desc(a + ks * 32), smem_desc(b + ks * 32), idesc,
                             (kt | p | ks) != 0 ? 1u : 0u);
            }
            mma_commit(&empty[s]);
        }
        mma_commit(&done);  // arrives once every MMA issued above has completed
    }
    __syncwarp();

    // epilogue: accumulator row (TMEM lane) = tile row; staged through shared
    // memory (the stage ring is idle once `done` has arrived)
    // block-uniform: tcgen05.ld below is warp-collective
    const bool ok = __syncthreads_and(mbar_wait(&done, 0) ? 1 : 0) != 0;
    tc_fence_after();
    float* stile = reinterpret_cast<float*>(smem);
    const int ld = P.bn + 1;
    if (ok) {
        const int row = warp * 32 + lane;
        const int r = m0 + row;
        const int pair = r >> 2, q = r & 3;
        const int z = 4 * (pair / P.na) + q;
        const float sc = pair < P.pairs ? row_scale(P.stats, z, P.nz, P.denorm, P.scale) : 0.0f;
        for (int c0 = 0; c0 < P.bn; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + (static_cast<unsigned>(warp * 32) << 16) + static_cast<unsigned>(c0), v);
#pragma unroll
            for (int i = 0; i < 16; ++i) stile[row * ld + c0 + i] = v[i] * sc;
        }
    } else if (threadIdx.x == 0) {
        atomicOr(err, 16u);
    }
    tc_fence_before();
    __syncthreads();
    if (ok) {
        const int npairs = BM / 4;
        const int pair0 = m0 >> 2;
        for (int idx = threadIdx.x; idx < npairs * P.bn; idx += blockDim.x) {
            const int ar = idx / P.bn, c = idx - ar * P.bn;
            const int n = n0 + c, pair = pair0 + ar;
            if (n >= P.sq || pair >= P.pairs) continue;
            const float* s4 = stile + (4 * ar) * ld + c;
            P.filt[static_cast<long long>(pair) * P.pitch + P.guard + n] =
                make_float4(s4[0], s4[ld], s4[2 * ld], s4[3 * ld]);
        }
    }
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS)
                     : "memory");
}

// X rows in (slice group, angle, slice % 4) order, split into three BF16
// terms (x0 = bf16(x), x1 = bf16(x - x0), x2 = bf16(x - x0 - x1); the
// differences are exact in float); K padded with zeros to kpad, rows past the
// last slice zero. The terms are stored one after the other, rows x kpad each.
__global__ void __launch_bounds__(256) k_split_rows(const float* __restrict__ sino, int nz, int na, int nd,
                                                    int kpad, long long rows, __nv_bfloat16* __restrict__ x0) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long per_row = kpad / 8;
    if (i >= rows * per_row) return;
    const long long r = i / per_row;
    const int k0 = static_cast<int>(i - r * per_row) * 8;
    const int pair = static_cast<int>(r >> 2), q = static_cast<int>(r & 3);
    const int z = 4 * (pair / na) + q, a = pair % na;
    const float* src = sino + (static_cast<long long>(z) * na + a) * nd;
    __align__(16) __nv_bfloat16 term[NTERMS][8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int k = k0 + t;
        float x = (z < nz && k < nd) ? src[k] : 0.0f;
#pragma unroll
        for (int a = 0; a < NTERMS; ++a) {
            term[a][t] = __float2bfloat16_rn(x);
            x -= __bfloat162float(term[a][t]);
        }
    }
    const long long plane = rows * kpad;
#pragma unroll
    for (int a = 0; a < NTERMS; ++a)
        *reinterpret_cast<uint4*>(x0 + a * plane + r * kpad + k0) = *reinterpret_cast<const uint4*>(term[a]);
}

// Round-to-nearest-even float -> bf16 bits (finite inputs).
unsigned short bf16_bits(float f) {
    unsigned u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return static_cast<unsigned short>(u >> 16);
}
float bf16_value(unsigned short b) {
    const unsigned u = static_cast<unsigned>(b) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 2-D bf16 tensor map over rows x kpad, box of `box_rows` x 64 with the
// 128-byte swizzle (the shared layout the MMA descriptors describe).
bool encode_map(void* out, const void* base, long long rows, int kpad, int box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(kpad), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(kpad) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(BK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
                          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    std::memcpy(out, &m, sizeof m);
    return true;
}

}  // namespace

int gemm_kpad(int bins) { return (bins + BK - 1) / BK * BK; }

size_t filter_gemm_split_bytes(int nz, int na, int bins) {
    const long long rows = (static_cast<long long>((nz + 3) / 4) * na * 4 + BM - 1) / BM * BM;
    return static_cast<size_t>(rows) * gemm_kpad(bins) * NTERMS * sizeof(__nv_bfloat16);
}

cudaError_t make_gemm_table(const PadGeom& g, int type, bool keep_nyquist, GemmTable* out) {
    static_assert(sizeof(CUtensorMap) == sizeof(out->map[0]), "tensor map size");
    static_assert(sizeof(out->map) / sizeof(out->map[0]) == NTERMS, "one map per term");
    const int ntiles = (g.sq + BNMAX - 1) / BNMAX;
    const int bn = 16 * ((g.sq + 16 * ntiles - 1) / (16 * ntiles));
    const int nrows = ntiles * bn;
    const int kpad = gemm_kpad(g.bins);
    const std::vector<double> h = conv_kernel(g, type, keep_nyquist);
    const int dmin = -(g.pad + g.bins - 1);
    // T's three BF16 terms, each the rounding of what the previous ones leave
    // (in double), stored one after the other
    const size_t plane = static_cast<size_t>(nrows) * kpad;
    std::vector<unsigned short> tt(NTERMS * plane, 0);
    for (int i = 0; i < g.sq; ++i)
        for (int j = 0; j < g.bins; ++j) {
            double t = h[i - g.pad - j - dmin];
            for (int a = 0; a < NTERMS; ++a) {
                const unsigned short b = bf16_bits(static_cast<float>(t));
                tt[a * plane + static_cast<size_t>(i) * kpad + j] = b;
                t -= bf16_value(b);
            }
        }
    const size_t bytes = plane * 2;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, NTERMS * bytes);
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(p, tt.data(), NTERMS * bytes, cudaMemcpyHostToDevice);
    // a copy from pageable memory may return before its DMA lands; the kernels
    // that read the table run on other streams, so wait for it here
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    for (int a = 0; a < NTERMS && e == cudaSuccess; ++a)
        if (!encode_map(out->map[a], static_cast<char*>(p) + a * bytes, nrows, kpad, bn)) e = cudaErrorNotSupported;
    if (e != cudaSuccess) {
        cudaFree(p);
        return e;
    }
    out->T.ptr = p;
    out->T.bytes = NTERMS * bytes;
    out->bn = bn;
    out->ntiles = ntiles;
    out->nrows = nrows;
    out->kpad = kpad;
    return cudaSuccess;
}

cudaError_t launch_filter_gemm_prep(const float* d_sino, int nz, int na, const PadGeom& g, const FiltLayout& fl,
                                    const GemmTable& tab, float4* d_filt, void* d_split, cudaStream_t st) {
    const int nzg = (nz + 3) / 4;
    const long long pairs = static_cast<long long>(nzg) * na;
    const long long rows = (pairs * 4 + BM - 1) / BM * BM;
    if (rows / BM > 65535) return cudaErrorInvalidValue;
    __nv_bfloat16* x0 = static_cast<__nv_bfloat16*>(d_split);
    const long long items = rows * (tab.kpad / 8);
    k_split_rows<<<static_cast<unsigned>((items + 255) / 256), 256, 0, st>>>(d_sino, nz, na, g.bins, tab.kpad,
                                                                              rows, x0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // zero guard bins on both sides of every filtered row
    const size_t pitch_b = sizeof(float4) * fl.pitch;
    if (fl.guard > 0) {
        e = cudaMemset2DAsync(d_filt, pitch_b, 0, sizeof(float4) * fl.guard, pairs, st);
        if (e != cudaSuccess) return e;
    }
    const int right = fl.pitch - fl.guard - g.sq;
    if (right > 0) e = cudaMemset2DAsync(d_filt + fl.guard + g.sq, pitch_b, 0, sizeof(float4) * right, pairs, st);
    return e;
}

cudaError_t launch_filter_gemm(const float* d_sino, int nz, int na, const PadGeom& g, const FiltLayout& fl,
                               const GemmTable& tab, const float4* d_stats, int denorm, float scale,
                               float4* d_filt, void* d_split, unsigned* d_err, cudaStream_t st) {
    const int nzg = (nz + 3) / 4;
    const long long pairs = static_cast<long long>(nzg) * na;
    const long long rows = (pairs * 4 + BM - 1) / BM * BM;
    if (rows / BM > 65535 || pairs > 0x7fffffffLL) return cudaErrorInvalidValue;
    (void)d_sino;
    const __nv_bfloat16* x0 = static_cast<const __nv_bfloat16*>(d_split);
    cudaError_t e;
    GemmMaps maps;
    for (int a = 0; a < NTERMS; ++a) {
        if (!encode_map(&maps.x[a], x0 + a * rows * tab.kpad, rows, tab.kpad, BM)) return cudaErrorNotSupported;
        std::memcpy(&maps.t[a], tab.map[a], sizeof maps.t[a]);
    }
    GemmParams P;
    P.filt = d_filt;
    P.stats = d_stats;
    P.nz = nz;
    P.na = na;
    P.sq = g.sq;
    P.guard = fl.guard;
    P.pitch = fl.pitch;
    P.denorm = denorm;
    P.scale = scale;
    P.bn = tab.bn;
    P.nk = tab.kpad / BK;
    P.pairs = static_cast<int>(pairs);
    e = cudaFuncSetAttribute(k_filter_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (e != cudaSuccess) return e;
    const dim3 grid(tab.ntiles, static_cast<unsigned>(rows / BM));
    k_filter_gemm<<<grid, 128, SMEM_BYTES, st>>>(maps, P, d_err);
    return cudaGetLastError();
}

}  // namespace ctb
