// filter.cu — ramp filtering of sinogram rows (the filter stage of
// SerialBackend::reconstructSlice, SerialBackend.cpp:150-195).
//
// Per row the reference zero-pads the nd detector values to L = fft_size at
// offset pad_before, multiplies the real spectrum by H[k] (FilterDesign), and
// keeps the first square_bins samples of the inverse transform. Its inverse
// real FFT never reads the Nyquist bin (FFT.cpp:96 pairs bin 0 with bin 0), and
// H[0] = 0, so the effective spectrum is H[k] X[k] for 0 < k < L/2 and zero at
// k = 0 and k = L/2.
//
// Here two real rows travel as the real and imaginary parts of one complex
// sequence: with a real, even response the filtered rows come back as the real
// and imaginary parts of IFFT(Hs * FFT(row0 + i row1)). A block filters the four
// slices of a slice group at one angle (two complex FFTs of length L in shared
// memory, L/16 threads each). The FFT is a radix-16 Stockham transform (one
// radix-2/4/8 pass when log2 L is not a multiple of 4) with twiddles read
// from a double-precision-accurate table. Output rows are written as float4
// (one value per slice), the layout the backprojector stages, scaled by
// pi/(2 na) times the slice's denormalisation span.
#include <cmath>

#include "ctb_internal.h"

namespace ctb {
namespace {

// Shared-memory index padding: one float2 of padding per 16 keeps the
// stride-R accesses of the first pass free of bank conflicts.
__device__ __forceinline__ int padi(int p) { return p + (p >> 4); }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void dft2(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
    const float2 t0 = cadd(v0, v2), t1 = csub(v0, v2);
    const float2 t2 = cadd(v1, v3), t3 = mul_mi<INV>(csub(v1, v3));
    v0 = cadd(t0, t2);
    v2 = csub(t0, t2);
    v1 = cadd(t1, t3);
    v3 = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2* v) { dft4<INV>(v[0], v[1], v[2], v[3]); }

// exp(-+ 2 pi i m / 16) for m = 0..15 (cos, sin of multiples of pi/8)
__device__ __forceinline__ float2 w16(int m, bool inv) {
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    const float h = 0.70710678118654752440f;
    const float cs[16][2] = {{1.f, 0.f}, {c1, s1}, {h, h}, {s1, c1}, {0.f, 1.f}, {-s1, c1}, {-h, h},
                             {-c1, s1}, {-1.f, 0.f}, {-c1, -s1}, {-h, -h}, {-s1, -c1}, {0.f, -1.f},
                             {s1, -c1}, {h, -h}, {c1, -s1}};
    return make_float2(cs[m][0], inv ? cs[m][1] : -cs[m][1]);
}

template <bool INV>
__device__ __forceinline__ void dft8(float2* v) {
    float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft4<INV>(e);
    dft4<INV>(o);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 t = cmul(o[k], w16(2 * k, INV));
        v[k] = cadd(e[k], t);
        v[k + 4] = csub(e[k], t);
    }
}

template <bool INV>
__device__ __forceinline__ void dft16(float2* v) {
    // n = 4 n1 + n2, k = k1 + 4 k2
    float2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        y[n2][0] = v[n2];
        y[n2][1] = v[4 + n2];
        y[n2][2] = v[8 + n2];
        y[n2][3] = v[12 + n2];
        dft4<INV>(y[n2]);
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1)
            if (n2 > 0) y[n2][k1] = cmul(y[n2][k1], w16(n2 * k1, INV));
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        float2 z0 = y[0][k1], z1 = y[1][k1], z2 = y[2][k1], z3 = y[3][k1];
        dft4<INV>(z0, z1, z2, z3);
        v[k1] = z0;
        v[k1 + 4] = z1;
        v[k1 + 8] = z2;
        v[k1 + 12] = z3;
    }
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 2) dft2<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
    else dft16<INV>(v);
}

// One Stockham pass of radix R over a length-L sequence in shared memory,
// executed by T = L/(16 K) threads (16 K / R butterflies each). Ns is the
// length of the sub-transforms already combined. tw[i] = exp(-2 pi i i / L).
template <int R, bool INV, int K>
__device__ __forceinline__ void stockham_pass(float2* buf, int L, int Ns, int tid, int T,
                                              const float2* __restrict__ tw) {
    constexpr int NB = 16 * K / R;
    float2 v[NB][R];
    const int LR = L / R;
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
        const int j = tid + bi * T;
        const int k = j & (Ns - 1);
#pragma unroll
        for (int r = 0; r < R; ++r) v[bi][r] = buf[padi(j + r * LR)];
        if (Ns > 1) {
            const int step = L / (Ns * R);
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = __ldg(tw + r * k * step);
                if (INV) w.y = -w.y;
                v[bi][r] = cmul(v[bi][r], w);
            }
        }
        dft<R, INV>(v[bi]);
    }
    __syncthreads();
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
        const int j = tid + bi * T;
        const int k = j & (Ns - 1);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[padi(base + r * Ns)] = v[bi][r];
    }
    __syncthreads();
}

template <bool INV, int K>
__device__ void fft(float2* buf, int L, int logL, int tid, int T, const float2* __restrict__ tw) {
    int Ns = 1;
    const int rem = logL & 3;
    if (rem == 1) { stockham_pass<2, INV, K>(buf, L, Ns, tid, T, tw); Ns *= 2; }
    else if (rem == 2) { stockham_pass<4, INV, K>(buf, L, Ns, tid, T, tw); Ns *= 4; }
    else if (rem == 3) { stockham_pass<8, INV, K>(buf, L, Ns, tid, T, tw); Ns *= 8; }
    for (int p = 0; p < (logL >> 2); ++p) {
        stockham_pass<16, INV, K>(buf, L, Ns, tid, T, tw);
        Ns *= 16;
    }
}

// Per-slice output scale: pi/(2 na) times the denormalisation span.
__device__ __forceinline__ float slice_scale(const float4* stats, int z, int nz, int denorm,
                                             float scale) {
    if (z >= nz) return 0.0f;
    if (!stats || denorm == CTB_DENORM_NONE) return scale;
    const float4 st = stats[z];
    const float span = st.y - st.x;
    if (denorm == CTB_DENORM_SERIAL) return scale * (span <= 0.0f ? 1.0f : span);
    return span > 0.0f ? scale * span : 0.0f;  // OpenMP: span <= 0 -> min everywhere
}

// grid (na, nzg); block 2 * T threads with T = L / (16 K); dynamic smem
// 2 * (L + L/16) float2. K = 1 up to L = 4096, K = 2 for L = 8192.
template <int K>
__global__ void __launch_bounds__(512) k_filter(const float* __restrict__ sino, int nz, int na, int nd, int sq, int pad,
                         int L, int logL, int guard, int pitch, const float* __restrict__ Hs,
                         const float2* __restrict__ tw, const float4* __restrict__ stats,
                         int denorm, float scale, float4* __restrict__ filt) {
    extern __shared__ float2 smem[];
    const int a = blockIdx.x, zg = blockIdx.y;
    const int T = L / (16 * K);
    const int f = threadIdx.x / T;  // which of the two complex rows
    const int tid = threadIdx.x - f * T;
    const int lp = L + (L >> 4);
    float2* buf = smem + f * lp;
    // load rows (4zg + 2f) and (4zg + 2f + 1) as real and imaginary parts
    const int z0 = 4 * zg + 2 * f, z1 = z0 + 1;
    const float* r0 = sino + (static_cast<long long>(z0) * na + a) * nd;
    const float* r1 = sino + (static_cast<long long>(z1) * na + a) * nd;
    for (int i = tid; i < L; i += T) {
        const int j = i - pad;
        float re = 0.f, im = 0.f;
        if (j >= 0 && j < nd) {
            if (z0 < nz) re = __ldg(r0 + j);
            if (z1 < nz) im = __ldg(r1 + j);
        }
        buf[padi(i)] = make_float2(re, im);
    }
    __syncthreads();
    fft<false, K>(buf, L, logL, tid, T, tw);
    for (int k = tid; k < L; k += T) {
        const float h = __ldg(Hs + k);
        float2 v = buf[padi(k)];
        v.x *= h;
        v.y *= h;
        buf[padi(k)] = v;
    }
    __syncthreads();
    fft<true, K>(buf, L, logL, tid, T, tw);
    // write the first sq samples of all four rows as float4, guard bins as 0
    const float s0 = slice_scale(stats, 4 * zg + 0, nz, denorm, scale);
    const float s1 = slice_scale(stats, 4 * zg + 1, nz, denorm, scale);
    const float s2 = slice_scale(stats, 4 * zg + 2, nz, denorm, scale);
    const float s3 = slice_scale(stats, 4 * zg + 3, nz, denorm, scale);
    const float2* b0 = smem;
    const float2* b1 = smem + lp;
    float4* dst = filt + (static_cast<long long>(zg) * na + a) * pitch;
    for (int i = threadIdx.x; i < pitch; i += blockDim.x) {
        const int j = i - guard;
        float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j >= 0 && j < sq) {
            const float2 u = b0[padi(j)], v = b1[padi(j)];
            o = make_float4(u.x * s0, u.y * s1, v.x * s2, v.y * s3);
        }
        dst[i] = o;
    }
}

}  // namespace

cudaError_t launch_filter(const float* d_sino, int nz, int na, const PadGeom& g,
                          const FiltLayout& fl, const float* d_Hs, const float2* d_tw,
                          const float4* d_stats, int denorm, float scale, float4* d_filt,
                          cudaStream_t st) {
    int logL = 0;
    while ((1 << logL) < g.L) ++logL;
    const int K = g.L > 4096 ? 2 : 1;
    const int threads = 2 * (g.L / (16 * K));
    const size_t smem = 2 * static_cast<size_t>(g.L + (g.L >> 4)) * sizeof(float2);
    auto kern = K == 2 ? k_filter<2> : k_filter<1>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const dim3 grid(na, (nz + 3) / 4);
    kern<<<grid, threads, smem, st>>>(d_sino, nz, na, g.bins, g.sq, g.pad, g.L, logL, fl.guard,
                                      fl.pitch, d_Hs, d_tw, d_stats, denorm, scale, d_filt);
    return cudaGetLastError();
}

}  // namespace ctb
