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
// sequence: convolution with a real kernel is real-linear, so the filtered rows
// come back as the real and imaginary parts of IFFT(Hc * FFT(row0 + i row1)).
// The transform length is the convolution length Lc = nextPow2(sq + nd - 1)
// (about L/2) with the restricted-lag response Hc (conv_response): the same
// linear operator as the reference's length-L filtering. The rows sit at the
// start of the sequence (pad_before is folded into Hc's lag placement), so the
// upper half of the first pass's inputs is always zero. A block filters two
// slices at one angle (one complex FFT of length Lc in shared memory, Lc/16
// threads, Lc/32 past 4096). Blocks read their job from a job table, so one
// launch filters any number of sinogram stacks that share Lc. The FFT is a
// radix-16 Stockham transform (one
// radix-2/4/8 pass when log2 L is not a multiple of 4) with twiddles read
// from per-pass tables of correctly rounded values laid out so that the
// threads of a warp read consecutive entries (fft_twiddle_table); the packed
// kernel reads w^1, w^2, w^3 and w^4, w^8, w^12 of a butterfly and forms the
// other nine twiddles as one product each (tw_set). The last
// inverse pass writes its natural-order samples straight to the output rows, float4 per bin (one
// value per slice), the layout the backprojector stages, scaled by
// pi/(2 na) times the slice's denormalisation span.
#include <cmath>
#include <vector>

#include "ctb_internal.h"

namespace ctb {
namespace {

// float2 index of the packed copy of a table of n float2 (packed_offset)
__device__ __forceinline__ long long packed_offset_d(long long n) { return (n + 1) & ~1LL; }

// Shared-memory index padding: one float2 of padding per 16 keeps the
// stride-R accesses of the first pass free of bank conflicts.
__device__ __forceinline__ int padi(int p) { return p + (p >> 4); }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
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

// DFTs whose inputs R/2 .. R-1 are zero (the first pass, see first_pass): the
// first butterfly stage adds nothing, so it is left out. Same values as dft<R>
// on the zero-padded inputs.
template <bool INV>
__device__ __forceinline__ void dft4_half(float2& v0, float2& v1, float2& v2, float2& v3) {
    const float2 a = v0, b = v1;  // v2 = v3 = 0 on entry
    const float2 t3 = mul_mi<INV>(b);
    v0 = cadd(a, b);
    v2 = csub(a, b);
    v1 = cadd(a, t3);
    v3 = csub(a, t3);
}

template <int R, bool INV>
__device__ __forceinline__ void dft_half(float2* v) {
    if constexpr (R == 2) {
        v[1] = v[0];
    } else if constexpr (R == 4) {
        dft4_half<INV>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        float2 e0 = v[0], e1 = v[2], e2, e3, o0 = v[1], o1 = v[3], o2, o3;
        dft4_half<INV>(e0, e1, e2, e3);
        dft4_half<INV>(o0, o1, o2, o3);
        const float2 e[4] = {e0, e1, e2, e3}, o[4] = {o0, o1, o2, o3};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 t = cmul(o[k], w16(2 * k, INV));
            v[k] = cadd(e[k], t);
            v[k + 4] = csub(e[k], t);
        }
    } else {
        // n = 4 n1 + n2, k = k1 + 4 k2; inputs with n1 >= 2 are zero
        float2 y[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
            y[n2][0] = v[n2];
            y[n2][1] = v[4 + n2];
            dft4_half<INV>(y[n2][0], y[n2][1], y[n2][2], y[n2][3]);
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
}

// Twiddle tables. A Stockham pass of radix R that combines sub-transforms of
// length Ns multiplies input r of butterfly k (k = j mod Ns) by
// w = exp(-2 pi i r k / (Ns R)) (the conjugate in the inverse transform). The
// values of one (R, Ns) pair are stored r-major, entry (r - 1) Ns + k, so the
// lanes of a warp (consecutive j, hence consecutive k) read consecutive
// entries. Radix-16 tables for every Ns = 2^i < L/16 ... L/16 sit at
// 15 (Ns - 1); the table of a radix-2/4/8 last pass (Ns = L/R) follows at
// 15 (L/8 - 1). Both transforms of a row use the same tables.
__device__ __forceinline__ int tw16_offset(int Ns) { return 15 * (Ns - 1); }
__device__ __forceinline__ int twr_offset(int L) { return 15 * (L / 8 - 1); }

template <bool INV>
__device__ __forceinline__ float2 twiddle_mul(float2 v, float2 w) {
    return INV ? cmulc(v, w) : cmul(v, w);
}

// The twiddles w^r, r = 1 .. R-1, of one butterfly from a table laid out
// r-major with stride `st`: w^1, w^2, w^3 and w^4, w^8, w^12 (radix 16; w^4
// for radix 8) are read, the others formed as w^(4a) w^b, one product each.
template <int R>
__device__ __forceinline__ void tw_set_s(const float2* __restrict__ t, int st, float2 (&w)[16]) {
    w[1] = __ldg(t);
    if constexpr (R >= 4) {
        w[2] = __ldg(t + st);
        w[3] = __ldg(t + 2 * st);
    }
    if constexpr (R >= 8) {
        w[4] = __ldg(t + 3 * st);
        if constexpr (R == 16) {
            w[8] = __ldg(t + 7 * st);
            w[12] = __ldg(t + 11 * st);
        }
#pragma unroll
        for (int a = 4; a < R; a += 4) {
            w[a + 1] = cmul(w[a], w[1]);
            w[a + 2] = cmul(w[a], w[2]);
            w[a + 3] = cmul(w[a], w[3]);
        }
    }
}

// One Stockham pass of radix R over a length-L sequence in shared memory,
// executed by T = L/(16 K) threads (16 K / R butterflies each). Ns is the
// length of the sub-transforms already combined; tw holds the twiddle tables.
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
            static_assert(R == 16, "inner passes are radix 16");
            float2 w[16];
            tw_set_s<16>(tw + tw16_offset(Ns) + k, Ns, w);
#pragma unroll
            for (int r = 1; r < 16; ++r) v[bi][r] = twiddle_mul<INV>(v[bi][r], w[r]);
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

// Where the last inverse pass stores: sample e of the filtered row pair goes
// to dst[2 (guard + e)] scaled by (s0, s1) when e < sq; the others are dropped.
struct RowOut {
    float2* dst;
    int guard, sq;
    float s0, s1;
};

// The last inverse pass (Ns = L / R): its Stockham output is in natural order,
// sample j + r L/R in register r of butterfly j, so it is written straight to
// the filtered row instead of back to shared memory (coalesced over j).
template <int R, int K>
__device__ __forceinline__ void last_pass_out(const float2* buf, int L, int tid, int T,
                                              const float2* __restrict__ tw, const RowOut& o) {
    constexpr int NB = 16 * K / R;
    const int LR = L / R;  // = Ns
    float2 v[NB][R];
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
        const int j = tid + bi * T;
#pragma unroll
        for (int r = 0; r < R; ++r) v[bi][r] = buf[padi(j + r * LR)];
        if (LR > 1) {
            float2 w[16];
            tw_set_s<R>(tw + (R == 16 ? tw16_offset(LR) : twr_offset(L)) + j, LR, w);
#pragma unroll
            for (int r = 1; r < R; ++r) v[bi][r] = cmulc(v[bi][r], w[r]);
        }
        dft<R, true>(v[bi]);
        // sq = ceil(sqrt2 nd) and Lc >= sq + nd - 1 give sq <= 0.586 Lc + 1, so
        // outputs r >= RKEEP (positions >= sq) are never kept: the compiler
        // drops their arithmetic
        constexpr int RKEEP = R == 2 ? 2 : R == 4 ? 3 : R == 8 ? 5 : 10;
#pragma unroll
        for (int r = 0; r < RKEEP; ++r) {
            const int e = j + r * LR;
            if (e < o.sq) o.dst[2 * (o.guard + e)] = make_float2(v[bi][r].x * o.s0, v[bi][r].y * o.s1);
        }
    }
}

// First forward pass (Ns = 1): the inputs come straight from the two sinogram
// rows, which sit at the start of the sequence (positions [0, nd), zero
// beyond; the kernel's lags are placed to match, conv_response), so the
// zero-padded sequence is never materialised. Since Lc >= sq + nd - 1 >= 2 nd - 1
// and Lc is even, nd <= Lc/2: inputs r >= R/2 of every butterfly (positions
// j + r L/R >= L/2) are zero and the butterflies start from half their inputs.
template <int R, int K>
__device__ __forceinline__ void first_pass(float2* buf, int L, int tid, int T, const float* r0,
                                           const float* r1, int nd) {
    constexpr int NB = 16 * K / R;
    float2 v[NB][R];
    const int LR = L / R;
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
        const int j = tid + bi * T;
#pragma unroll
        for (int r = 0; r < R / 2; ++r) {
            const int i = j + r * LR;
            const bool in = i < nd;
            v[bi][r] = make_float2(in && r0 ? __ldg(r0 + i) : 0.0f, in && r1 ? __ldg(r1 + i) : 0.0f);
        }
        dft_half<R, false>(v[bi]);
    }
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
        const int j = tid + bi * T;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[padi(j * R + r)] = v[bi][r];
    }
    __syncthreads();
}

// The forward transform's last radix-16 pass (Ns = L/16) leaves spectrum bin
// j + r L/16 in register r of butterfly j -- exactly the inputs of the inverse
// transform's first radix-16 pass (Ns = 1). Both passes and the filter
// multiply between them run in registers.
template <int K>
__device__ __forceinline__ void fused_middle(float2* buf, int L, int tid, int T,
                                             const float2* __restrict__ tw,
                                             const float2* __restrict__ Hc) {
    constexpr int NB = K;
    float2 v[NB][16];
    const int LR = L / 16;
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
        const int j = tid + bi * T;
#pragma unroll
        for (int r = 0; r < 16; ++r) v[bi][r] = buf[padi(j + r * LR)];
        if (LR > 1) {
            float2 w[16];
            tw_set_s<16>(tw + tw16_offset(LR) + j, LR, w);
#pragma unroll
            for (int r = 1; r < 16; ++r) v[bi][r] = cmul(v[bi][r], w[r]);
        }
        dft16<false>(v[bi]);
#pragma unroll
        for (int r = 0; r < 16; ++r) v[bi][r] = cmul(v[bi][r], __ldg(Hc + j + r * LR));
        dft16<true>(v[bi]);
    }
    __syncthreads();
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
        const int j = tid + bi * T;
#pragma unroll
        for (int r = 0; r < 16; ++r) buf[padi(j * 16 + r)] = v[bi][r];
    }
    __syncthreads();
}

// Filter one complex row pair in shared memory: forward FFT, Hc multiply,
// inverse FFT (natural order out). Radix-16 passes around the fused middle; the
// radix-2/4/8 remainder pass runs first in the forward and last in the inverse.
template <int K>
__device__ void filter_rows(float2* buf, int L, int logL, int tid, int T, const float* r0,
                            const float* r1, int nd, const float2* __restrict__ tw,
                            const float2* __restrict__ Hc, const RowOut& out) {
    const int rem = logL & 3;
    const int q = logL >> 2;  // radix-16 passes per transform (>= 1 for L >= 64)
    int Ns = 1;
    if (rem == 1) { first_pass<2, K>(buf, L, tid, T, r0, r1, nd); Ns = 2; }
    else if (rem == 2) { first_pass<4, K>(buf, L, tid, T, r0, r1, nd); Ns = 4; }
    else if (rem == 3) { first_pass<8, K>(buf, L, tid, T, r0, r1, nd); Ns = 8; }
    else { first_pass<16, K>(buf, L, tid, T, r0, r1, nd); Ns = 16; }
    const int fwd16 = q - 1 - (rem == 0 ? 1 : 0);  // radix-16 passes between first and middle
    for (int p = 0; p < fwd16; ++p) {
        stockham_pass<16, false, K>(buf, L, Ns, tid, T, tw);
        Ns *= 16;
    }
    fused_middle<K>(buf, L, tid, T, tw, Hc);
    Ns = 16;
    // the inverse radix-16 passes; the last pass of the transform stores the
    // filtered rows itself
    const int inv16 = q - 1 - (rem == 0 ? 1 : 0);
    for (int p = 0; p < inv16; ++p) {
        stockham_pass<16, true, K>(buf, L, Ns, tid, T, tw);
        Ns *= 16;
    }
    if (rem == 1) last_pass_out<2, K>(buf, L, tid, T, tw, out);
    else if (rem == 2) last_pass_out<4, K>(buf, L, tid, T, tw, out);
    else if (rem == 3) last_pass_out<8, K>(buf, L, tid, T, tw, out);
    else if (q > 1) last_pass_out<16, K>(buf, L, tid, T, tw, out);
    else {
        // L = 16: the fused middle pass was the whole transform (natural order in buf)
        for (int e = tid; e < L; e += T)
            if (e < out.sq) {
                const float2 u = buf[padi(e)];
                out.dst[2 * (out.guard + e)] = make_float2(u.x * out.s0, u.y * out.s1);
            }
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
    if (denorm == CTB_DENORM_CUDA) return span > 0.0f ? scale * span : scale;
    return span > 0.0f ? scale * span : 0.0f;  // OpenMP: span <= 0 -> min everywhere
}

// One CTA per item (slice pair zp, angle a) of a job of the batch; block
// T = Lc/(16 K) threads filter slices 2 zp and 2 zp + 1 at angle a; dynamic smem
// (Lc + Lc/16) float2. An item's arithmetic depends only on its own job. With
// K = 1 the registers are held to 80 (three 256-thread or six 128-thread CTAs
// per SM), which measured faster than the compiler's own allocation.
template <int K>
__global__ void __launch_bounds__(256, (K == 1 ? 3 : 1)) k_filter(const __grid_constant__ FiltBatch batch, int logL) {
    extern __shared__ float2 smem[];
    const long long item = blockIdx.x + static_cast<long long>(blockIdx.y) * gridDim.x;
    if (item >= batch.total) return;
    int jb = 0;
    while (jb + 1 < batch.njobs && batch.job[jb + 1].first <= item) ++jb;
    const FiltJob& J = batch.job[jb];
    const long long local = item - J.first;
    const int na = J.na, nz = J.nz, nd = J.bins;
    const int a = static_cast<int>(local % na);
    const int z0 = 2 * static_cast<int>(local / na), z1 = z0 + 1;
    const int T = blockDim.x;
    const int tid = threadIdx.x;
    const float* r0 = J.sino + (static_cast<long long>(z0) * na + a) * nd;
    const float* r1 = z1 < nz ? J.sino + (static_cast<long long>(z1) * na + a) * nd : nullptr;
    // rows z0, z1 are lanes (z0 % 4, z0 % 4 + 1) of the float4 layout
    const int pitch = J.pitch, guard = J.guard, sq = J.sq;
    float2* dst = reinterpret_cast<float2*>(J.filt + (static_cast<long long>(z0 / 4) * na + a) * pitch) +
                  ((z0 & 3) >> 1);
    const RowOut out{dst, guard, sq, slice_scale(J.stats, z0, nz, J.denorm, J.scale),
                     slice_scale(J.stats, z1, nz, J.denorm, J.scale)};
    // guard bins on both sides of the row are zeros
    for (int i = tid; i < pitch - sq; i += T) {
        const int b = i < guard ? i : i + sq;
        dst[2 * b] = make_float2(0.f, 0.f);
    }
    filter_rows<K>(smem, batch.Lc, logL, tid, T, r0, r1, nd, batch.tw, J.Hc, out);
}

// ------------------------------------------------- two sequences per thread
// k_filter4 transforms two complex sequences in lockstep: A = row z0 + i row
// z0+1 and B = row z0+2 + i row z0+3 of one angle, i.e. the four slices of one
// float4 group of the filtered-row layout. A C2 value holds one element of
// each, (re_A, re_B) and (im_A, im_B), so every complex add or multiply of the
// FFT is one packed FP32x2 instruction (FADD2 / FMUL2 / FFMA2) on the pair,
// shared memory moves one float4 per element pair, and the output is written
// as whole float4 bins. Each lane of a packed instruction rounds exactly as
// the scalar one, and the operations and their order are those of the scalar
// butterflies above, so each sequence is transformed exactly as the scalar
// kernel would transform it. The transform length is a template parameter:
// every pass, stride and table offset is a compile-time constant.
struct C2 {
    float2 re, im;
};

__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b in one instruction: fma(b, -1, a) rounds a - b exactly once
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ C2 c2add(C2 a, C2 b) { return C2{p_add(a.re, b.re), p_add(a.im, b.im)}; }
__device__ __forceinline__ C2 c2sub(C2 a, C2 b) { return C2{p_sub(a.re, b.re), p_sub(a.im, b.im)}; }
// a * (c + i s) with the rounding of cmul: cc = (c, c), ss = (s, s), nss = -ss
__device__ __forceinline__ C2 c2mul(C2 a, float2 cc, float2 ss, float2 nss) {
    return C2{__ffma2_rn(a.re, cc, __fmul2_rn(a.im, nss)), __ffma2_rn(a.re, ss, __fmul2_rn(a.im, cc))};
}
// a * conj(c + i s) with the rounding of cmulc
__device__ __forceinline__ C2 c2mulc(C2 a, float2 cc, float2 ss, float2 nss) {
    return C2{__ffma2_rn(a.re, cc, __fmul2_rn(a.im, ss)), __ffma2_rn(a.im, cc, __fmul2_rn(a.re, nss))};
}
// multiplication by the constant w16(m) (exp(-+ 2 pi i m / 16))
template <bool INV>
__device__ __forceinline__ C2 c2mul16(C2 a, int m) {
    const float2 w = w16(m, INV);
    return c2mul(a, make_float2(w.x, w.x), make_float2(w.y, w.y), make_float2(-w.y, -w.y));
}

// dft4 on pairs; the factor -+i is applied by choosing add or subtract per
// component (t1 +- (-+i) d), which rounds as the scalar cadd of mul_mi.
template <bool INV>
__device__ __forceinline__ void dft4p(C2& v0, C2& v1, C2& v2, C2& v3) {
    const C2 t0 = c2add(v0, v2), t1 = c2sub(v0, v2);
    const C2 t2 = c2add(v1, v3), d = c2sub(v1, v3);
    v0 = c2add(t0, t2);
    v2 = c2sub(t0, t2);
    if (!INV) {  // t3 = -i d = (d.im, -d.re)
        v1 = C2{p_add(t1.re, d.im), p_sub(t1.im, d.re)};
        v3 = C2{p_sub(t1.re, d.im), p_add(t1.im, d.re)};
    } else {  // t3 = +i d = (-d.im, d.re)
        v1 = C2{p_sub(t1.re, d.im), p_add(t1.im, d.re)};
        v3 = C2{p_add(t1.re, d.im), p_sub(t1.im, d.re)};
    }
}
// dft4p with v2 = v3 = 0 on entry (the first stage of a half-input DFT)
template <bool INV>
__device__ __forceinline__ void dft4p_half(C2& v0, C2& v1, C2& v2, C2& v3) {
    const C2 a = v0, d = v1;
    v0 = c2add(a, d);
    v2 = c2sub(a, d);
    if (!INV) {
        v1 = C2{p_add(a.re, d.im), p_sub(a.im, d.re)};
        v3 = C2{p_sub(a.re, d.im), p_add(a.im, d.re)};
    } else {
        v1 = C2{p_sub(a.re, d.im), p_add(a.im, d.re)};
        v3 = C2{p_add(a.re, d.im), p_sub(a.im, d.re)};
    }
}

template <bool INV, bool HALF>
__device__ __forceinline__ void dft8p(C2* v) {
    C2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    if (HALF) {
        dft4p_half<INV>(e[0], e[1], e[2], e[3]);
        dft4p_half<INV>(o[0], o[1], o[2], o[3]);
    } else {
        dft4p<INV>(e[0], e[1], e[2], e[3]);
        dft4p<INV>(o[0], o[1], o[2], o[3]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const C2 t = c2mul16<INV>(o[k], 2 * k);
        v[k] = c2add(e[k], t);
        v[k + 4] = c2sub(e[k], t);
    }
}

template <bool INV, bool HALF>
__device__ __forceinline__ void dft16p(C2* v) {
    C2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        y[n2][0] = v[n2];
        y[n2][1] = v[4 + n2];
        if (HALF) {
            dft4p_half<INV>(y[n2][0], y[n2][1], y[n2][2], y[n2][3]);
        } else {
            y[n2][2] = v[8 + n2];
            y[n2][3] = v[12 + n2];
            dft4p<INV>(y[n2][0], y[n2][1], y[n2][2], y[n2][3]);
        }
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1)
            if (n2 > 0) y[n2][k1] = c2mul16<INV>(y[n2][k1], n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        C2 z0 = y[0][k1], z1 = y[1][k1], z2 = y[2][k1], z3 = y[3][k1];
        dft4p<INV>(z0, z1, z2, z3);
        v[k1] = z0;
        v[k1 + 4] = z1;
        v[k1 + 8] = z2;
        v[k1 + 12] = z3;
    }
}

template <int R, bool INV, bool HALF = false>
__device__ __forceinline__ void dftp(C2* v) {
    if constexpr (R == 2) {
        if (HALF) {
            v[1] = v[0];
        } else {
            const C2 a = v[0], b = v[1];
            v[0] = c2add(a, b);
            v[1] = c2sub(a, b);
        }
    } else if constexpr (R == 4) {
        if (HALF) dft4p_half<INV>(v[0], v[1], v[2], v[3]);
        else dft4p<INV>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        dft8p<INV, HALF>(v);
    } else {
        dft16p<INV, HALF>(v);
    }
}

// Shared-memory element p (a float4: one C2) lives at p ^ f(p >> 3),
// f(q) = (q + q / 8) mod 8: a permutation inside every group of 8 elements
// that keeps the 8 lanes of each LDS.128/STS.128 phase on distinct banks for
// the unit, 8 and 16 strides of the passes at every length from 64 to 2048
// except one pass at 512 and 1024 (two-way).
__device__ __forceinline__ int swz(int p) { return p ^ (((p >> 3) + (p >> 6)) & 7); }
__device__ __forceinline__ C2 ld_c2(const float4* buf, int p) {
    const float4 t = buf[swz(p)];
    return C2{make_float2(t.x, t.y), make_float2(t.z, t.w)};
}
__device__ __forceinline__ void st_c2(float4* buf, int p, C2 v) {
    buf[swz(p)] = make_float4(v.re.x, v.re.y, v.im.x, v.im.y);
}
// twiddle from the packed table: w = {wx, wx, wy, wy}
template <bool INV>
__device__ __forceinline__ C2 c2tw(C2 v, float4 w) {
    const float2 cc = make_float2(w.x, w.y), ss = make_float2(w.z, w.w);
    const float2 nss = __fmul2_rn(ss, make_float2(-1.0f, -1.0f));
    return INV ? c2mulc(v, cc, ss, nss) : c2mul(v, cc, ss, nss);
}

// Product of two packed twiddles {c, c, s, s}; nq = {-s, -s} of q.
__device__ __forceinline__ float4 tw_mul(float4 p, float4 q, float2 nq) {
    const float2 c1 = make_float2(p.x, p.y), s1 = make_float2(p.z, p.w);
    const float2 c2 = make_float2(q.x, q.y), s2 = make_float2(q.z, q.w);
    const float2 cc = __ffma2_rn(s1, nq, __fmul2_rn(c1, c2));
    const float2 ss = __ffma2_rn(c1, s2, __fmul2_rn(s1, c2));
    return make_float4(cc.x, cc.y, ss.x, ss.y);
}
// The twiddles w^r, r = 1 .. R-1, of one butterfly from a packed table laid out
// r-major with stride `st` (entry (r - 1) st): w^1, w^2, w^3 and the powers
// w^4, w^8, w^12 (radix 16; w^4 for radix 8) are read, the others formed as
// w^(4a) w^b (a one product from two correctly rounded values, ~1.5 ulp), so
// a pass reads 6 of its 15 table entries (4 of 7 at radix 8).
template <int R>
__device__ __forceinline__ void tw_set(const float4* __restrict__ t, int st, float4 (&w)[16]) {
    w[1] = __ldg(t);
    if constexpr (R >= 4) {
        w[2] = __ldg(t + st);
        w[3] = __ldg(t + 2 * st);
    }
    if constexpr (R >= 8) {
        w[4] = __ldg(t + 3 * st);
        const float2 n1 = make_float2(-w[1].z, -w[1].w), n2 = make_float2(-w[2].z, -w[2].w),
                     n3 = make_float2(-w[3].z, -w[3].w);
        if constexpr (R == 16) {
            w[8] = __ldg(t + 7 * st);
            w[12] = __ldg(t + 11 * st);
        }
#pragma unroll
        for (int a = 4; a < R; a += 4) {
            w[a + 1] = tw_mul(w[a], w[1], n1);
            w[a + 2] = tw_mul(w[a], w[2], n2);
            w[a + 3] = tw_mul(w[a], w[3], n3);
        }
    }
}

// One radix-16 Stockham pass (Ns > 1) of length L by T = L/16 threads.
template <int L, int NS, bool INV>
__device__ __forceinline__ void pass16p(float4* buf, int j, const float4* __restrict__ tw4) {
    constexpr int LR = L / 16;
    const int k = j & (NS - 1);
    C2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = ld_c2(buf, j + r * LR);
    float4 w[16];
    tw_set<16>(tw4 + 15 * (NS - 1) + k, NS, w);
#pragma unroll
    for (int r = 1; r < 16; ++r) v[r] = c2tw<INV>(v[r], w[r]);
    dftp<16, INV>(v);
    __syncthreads();
    const int base = (j - k) * 16 + k;
#pragma unroll
    for (int r = 0; r < 16; ++r) st_c2(buf, base + r * NS, v[r]);
    __syncthreads();
}

// The forward radix-16 passes after the first (compile-time recursion over Ns).
template <int L, int NS, int LEFT, bool INV>
__device__ __forceinline__ void passes16p(float4* buf, int j, const float4* __restrict__ tw4) {
    if constexpr (LEFT > 0) {
        pass16p<L, NS, INV>(buf, j, tw4);
        passes16p<L, NS * 16, LEFT - 1, INV>(buf, j, tw4);
    }
}

// Lengths up to kPackedMaxL = 2048, registers held to 128 (four CTAs per SM
// at 2048, no spills; a 96-register cap for a fifth CTA spills and measured
// slower, 1.81 against 1.56 ms at 512^3 x 720). At 4096 the 16 pairs per
// thread need more than 128 registers (one 256-thread CTA per SM) and the
// kernel is slower than the scalar one (5.35 against 4.68 ms at 1024^2 x 256 x
// 1440), which therefore keeps lengths 4096 and 8192.
template <int LOGL>
__global__ void __launch_bounds__((1 << LOGL) / 16, 4) k_filter4(const __grid_constant__ FiltBatch batch) {
    constexpr int L = 1 << LOGL, T = L / 16, REM = LOGL & 3, Q = LOGL >> 2;
    constexpr int R0 = REM ? (1 << REM) : 16;  // radix of the first and the last pass
    constexpr int NB0 = 16 / R0;               // their butterflies per thread
    constexpr int FWD16 = Q - 1 - (REM == 0 ? 1 : 0);
    extern __shared__ float4 smem4[];
    const long long item = blockIdx.x + static_cast<long long>(blockIdx.y) * gridDim.x;
    if (item >= batch.total) return;
    int jb = 0;
    while (jb + 1 < batch.njobs && batch.job[jb + 1].first <= item) ++jb;
    const FiltJob& J = batch.job[jb];
    const long long local = item - J.first;
    const int na = J.na, nz = J.nz, nd = J.bins, sq = J.sq, guard = J.guard, pitch = J.pitch;
    const int a = static_cast<int>(local % na);
    const int zg = static_cast<int>(local / na);
    const int z0 = 4 * zg;
    const int tid = threadIdx.x;
    const float* rows[4];
#pragma unroll
    for (int s = 0; s < 4; ++s)
        rows[s] = z0 + s < nz ? J.sino + (static_cast<long long>(z0 + s) * na + a) * nd : nullptr;
    const float4* tw4 = reinterpret_cast<const float4*>(batch.tw + packed_offset_d(batch.twlen));
    const float4* Hc4 = reinterpret_cast<const float4*>(J.Hc + L);
    float4* dst = J.filt + (static_cast<long long>(zg) * na + a) * pitch;
    // guard bins on both sides of the row are zeros
    for (int i = tid; i < pitch - sq; i += T) dst[i < guard ? i : i + sq] = make_float4(0.f, 0.f, 0.f, 0.f);

    // first forward pass (Ns = 1): the rows sit at positions [0, nd) with
    // nd <= L/2, so inputs r >= R0/2 of every butterfly are zero
    {
        constexpr int LR = L / R0;
#pragma unroll
        for (int bi = 0; bi < NB0; ++bi) {
            const int j = tid + bi * T;
            C2 v[R0];
#pragma unroll
            for (int r = 0; r < R0 / 2; ++r) {
                const int i = j + r * LR;
                const bool in = i < nd;
                v[r].re = make_float2(in && rows[0] ? __ldg(rows[0] + i) : 0.0f, in && rows[2] ? __ldg(rows[2] + i) : 0.0f);
                v[r].im = make_float2(in && rows[1] ? __ldg(rows[1] + i) : 0.0f, in && rows[3] ? __ldg(rows[3] + i) : 0.0f);
            }
            dftp<R0, false, true>(v);
#pragma unroll
            for (int r = 0; r < R0; ++r) st_c2(smem4, j * R0 + r, v[r]);
        }
        __syncthreads();
    }
    passes16p<L, R0, FWD16, false>(smem4, tid, tw4);
    // the forward transform's last radix-16 pass (Ns = L/16), the filter
    // multiply and the inverse transform's first radix-16 pass (Ns = 1), all in
    // registers
    {
        constexpr int LR = L / 16;
        const int j = tid;
        C2 v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = ld_c2(smem4, j + r * LR);
        if constexpr (LR > 1) {
            float4 w[16];
            tw_set<16>(tw4 + 15 * (LR - 1) + j, LR, w);
#pragma unroll
            for (int r = 1; r < 16; ++r) v[r] = c2tw<false>(v[r], w[r]);
        }
        dftp<16, false>(v);
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const float4 h = __ldg(Hc4 + j + r * LR);
            v[r] = c2mul(v[r], make_float2(h.x, h.y), make_float2(h.z, h.w),
                         __fmul2_rn(make_float2(h.z, h.w), make_float2(-1.0f, -1.0f)));
        }
        dftp<16, true>(v);
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 16; ++r) st_c2(smem4, j * 16 + r, v[r]);
        __syncthreads();
    }
    passes16p<L, 16, FWD16, true>(smem4, tid, tw4);
    // the last inverse pass (Ns = L / R0) stores the filtered bins: position e
    // of the row pair is bin e, kept when e < sq (and sq <= 0.586 L + 1, so
    // outputs r >= RKEEP never are)
    {
        constexpr int LR = L / R0;
        constexpr int RKEEP = R0 == 2 ? 2 : R0 == 4 ? 3 : R0 == 8 ? 5 : 10;
        const float s0 = slice_scale(J.stats, z0, nz, J.denorm, J.scale);
        const float s1 = slice_scale(J.stats, z0 + 1, nz, J.denorm, J.scale);
        const float s2 = slice_scale(J.stats, z0 + 2, nz, J.denorm, J.scale);
        const float s3 = slice_scale(J.stats, z0 + 3, nz, J.denorm, J.scale);
        const float2 sre = make_float2(s0, s2), sim = make_float2(s1, s3);
#pragma unroll
        for (int bi = 0; bi < NB0; ++bi) {
            const int j = tid + bi * T;
            C2 v[R0];
#pragma unroll
            for (int r = 0; r < R0; ++r) v[r] = ld_c2(smem4, j + r * LR);
            if constexpr (LR > 1) {
                float4 w[16];
                tw_set<R0>(tw4 + (R0 == 16 ? 15 * (LR - 1) : 15 * (L / 8 - 1)) + j, LR, w);
#pragma unroll
                for (int r = 1; r < R0; ++r) v[r] = c2tw<true>(v[r], w[r]);
            }
            dftp<R0, true>(v);
#pragma unroll
            for (int r = 0; r < RKEEP; ++r) {
                const int e = j + r * LR;
                if (e < sq) {
                    const float2 re = __fmul2_rn(v[r].re, sre), im = __fmul2_rn(v[r].im, sim);
                    dst[guard + e] = make_float4(re.x, im.x, re.y, im.y);
                }
            }
        }
    }
}

}  // namespace

size_t fft_twiddle_len(int L) {
    int logL = 0;
    while ((1 << logL) < L) ++logL;
    const int rem = logL & 3;
    const size_t n16 = 15 * static_cast<size_t>(L / 8 - 1);  // radix-16 tables, Ns = 1 .. L/16
    return rem == 0 ? n16 : n16 + static_cast<size_t>((1 << rem) - 1) * (L >> rem);
}

std::vector<float2> fft_twiddle_table(int L) {
    const size_t n2 = fft_twiddle_len(L);
    std::vector<float2> t(n2, make_float2(1.0f, 0.0f));
    auto put = [&](size_t off, int R, int Ns) {
        for (int r = 1; r < R; ++r)
            for (int k = 0; k < Ns; ++k) {
                // exp(-2 pi i r k / (Ns R)), argument reduced exactly in integers
                const long long m = (static_cast<long long>(r) * k) % (static_cast<long long>(Ns) * R);
                const double a = 2.0 * 3.14159265358979323846 * static_cast<double>(m) / (static_cast<double>(Ns) * R);
                t[off + static_cast<size_t>(r - 1) * Ns + k] =
                    make_float2(static_cast<float>(std::cos(a)), static_cast<float>(-std::sin(a)));
            }
    };
    for (int Ns = 1; Ns <= L / 16; Ns *= 2) put(15 * static_cast<size_t>(Ns - 1), 16, Ns);
    int logL = 0;
    while ((1 << logL) < L) ++logL;
    const int rem = logL & 3;
    if (rem) put(15 * static_cast<size_t>(L / 8 - 1), 1 << rem, L >> rem);
    if (L <= kPackedMaxL) {
        // the packed copy for k_filter4: entry i as (wx, wx) (wy, wy), from a
        // 16-byte boundary (an even float2 index)
        t.resize(packed_offset(n2), make_float2(0.0f, 0.0f));
        for (size_t i = 0; i < n2; ++i) {
            t.push_back(make_float2(t[i].x, t[i].x));
            t.push_back(make_float2(t[i].y, t[i].y));
        }
    }
    return t;
}

std::vector<float2> filter_table(const PadGeom& g, int type, bool keep_nyquist) {
    const std::vector<double> Hd = conv_response(g, type, keep_nyquist);
    std::vector<float2> Hc(g.Lc);
    for (int k = 0; k < g.Lc; ++k)
        Hc[k] = make_float2(static_cast<float>(Hd[2 * k]), static_cast<float>(Hd[2 * k + 1]));
    if (g.Lc <= kPackedMaxL)
        for (int k = 0; k < g.Lc; ++k) {  // packed copy after the Lc entries
            const float2 h = Hc[k];
            Hc.push_back(make_float2(h.x, h.x));
            Hc.push_back(make_float2(h.y, h.y));
        }
    return Hc;
}

FiltJob make_filt_job(const float* d_sino, int nz, int na, const PadGeom& g, const FiltLayout& fl,
                      const float2* d_Hc, const float4* d_stats, int denorm, float scale,
                      float4* d_filt) {
    FiltJob J;
    J.sino = d_sino;
    J.filt = d_filt;
    J.stats = d_stats;
    J.Hc = d_Hc;
    J.nz = nz;
    J.na = na;
    J.bins = g.bins;
    J.sq = g.sq;
    J.pad = g.pad;
    J.guard = fl.guard;
    J.pitch = fl.pitch;
    J.denorm = denorm;
    J.scale = scale;
    J.first = 0;
    return J;
}

template <int LOGL>
cudaError_t launch_filter4(const FiltBatch& b, cudaStream_t st) {
    constexpr int L = 1 << LOGL;
    const size_t smem = sizeof(float4) * L;
    cudaError_t e = cudaFuncSetAttribute(k_filter4<LOGL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    // (no shared-memory carveout preference: the twiddle and spectrum tables
    // are read through L1, and a full carveout measured slower, 1.71 ms
    // against 1.56 ms at 512^3 x 720)
    if (e != cudaSuccess) return e;
    const long long gx = b.total < 65535 ? b.total : 65535;
    const long long gy = (b.total + gx - 1) / gx;
    if (gy > 65535) return cudaErrorInvalidValue;
    k_filter4<LOGL><<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(gy)), L / 16, smem, st>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_filter_batch(const FiltBatch& b, cudaStream_t st) {
    const int L = b.Lc;
    if (b.total == 0) return cudaSuccess;
    int logL = 0;
    while ((1 << logL) < L) ++logL;
    if (L <= kPackedMaxL) {
        // four slices (two sequences) per item: (slice group, angle) items
        FiltBatch p = b;
        p.twlen = static_cast<long long>(fft_twiddle_len(L));
        p.total = 0;
        for (int k = 0; k < p.njobs; ++k) {
            p.job[k].first = p.total;
            p.total += static_cast<long long>(p.job[k].na) * ((p.job[k].nz + 3) / 4);
        }
        static_assert(kPackedMaxL == 2048, "one instantiation per length up to kPackedMaxL");
        switch (logL) {
        case 6: return launch_filter4<6>(p, st);
        case 7: return launch_filter4<7>(p, st);
        case 8: return launch_filter4<8>(p, st);
        case 9: return launch_filter4<9>(p, st);
        case 10: return launch_filter4<10>(p, st);
        default: return launch_filter4<11>(p, st);
        }
    }
    const int K = L > 4096 ? 2 : 1;
    const int threads = L / (16 * K);
    const size_t smem = static_cast<size_t>(L + (L >> 4)) * sizeof(float2);
    auto kern = K == 2 ? k_filter<2> : k_filter<1>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    // items on a 2-D grid (x up to 65535 wide rows) so totals past 2^31 stay addressable
    const long long gx = b.total < 65535 ? b.total : 65535;
    const long long gy = (b.total + gx - 1) / gx;
    if (gy > 65535) return cudaErrorInvalidValue;
    kern<<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(gy)), threads, smem, st>>>(b, logL);
    return cudaGetLastError();
}

cudaError_t launch_filter(const float* d_sino, int nz, int na, const PadGeom& g,
                          const FiltLayout& fl, const float2* d_Hc, const float2* d_tw,
                          const float4* d_stats, int denorm, float scale, float4* d_filt,
                          cudaStream_t st) {
    FiltBatch b;
    b.njobs = 1;
    b.Lc = g.Lc;
    b.tw = d_tw;
    b.job[0] = make_filt_job(d_sino, nz, na, g, fl, d_Hc, d_stats, denorm, scale, d_filt);
    b.total = static_cast<long long>(na) * ((nz + 1) / 2);
    return launch_filter_batch(b, st);
}

}  // namespace ctb
