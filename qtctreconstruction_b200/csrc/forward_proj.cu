// forward_proj.cu — the forward projector (the RadonTransform stage of the
// FBP path).
//
// The reference's forward projector (SerialBackend::computeSinogram,
// SerialBackend.cpp:59-136) splats every non-zero pixel onto the two detector
// bins around s = (x-cx)cos + (y-cy)sin + floor(nd/2) with weights
// (1 - frac, frac), frac = s - floor(s). For bins 1 .. nd-2 that is the hat
// function: bin b = sum over pixels of v * max(0, 1 - |s - b|). Bins 0 and
// nd-1 follow the reference's own rules instead (a pixel with floor(s) = -1
// adds nothing to bin 0; floor(s) = nd-1 adds its full value to bin nd-1).
//
// Here a warp computes a strip of K consecutive output bins of one angle for
// 4 NP slices, walking the image along the axis the detector is closest to
// (rows when |cos| >= |sin|, else columns of the transposed copy). At walked
// row p the strip's pixels are the 32 consecutive columns from the crossing
// q*(p) of its lower bin edge: lane l owns column rint(q*) + S l (S the sign
// of ds/dq), whose offset from the crossing is u = (l - phi) |kq| in bins,
// phi = S (rint(q*) - q*) in [-1/2, 1/2]. So every row is one coalesced load
// of 32 neighbouring pixels (each the 8 slices of a plane pair, 32 bytes, one
// 256-bit load per lane), and lane l's pixel
// always falls in bin m_l or m_l + 1 of the strip, m_l = floor((l - 1/2)
// |kq|), whatever the row: the lane keeps three accumulators, for bins m_l,
// m_l + 1 and m_l + 2, adding v times the hat weights of its pixel. At the
// end of the walk the warp adds, per output bin, the accumulators of the few
// lanes that reach it, in lane order, gathered by warp shuffles. K is chosen per
// angle group so that K + 1 <= 31.5 |kq|: the lanes' pixels cover the
// strip's bins and the bin on either side.
//
// The crossing is evaluated in double once per chunk of PCH = 16 rows (an
// integer column plus a float offset) and stepped in float within the chunk;
// each 8-row half of a chunk is walked only where its lanes' columns meet the
// non-zero pixels of that 8-row band. The warps of a CTA are the up to GMAX =
// 4 angles of a group that share the walked axis, on the same strip index;
// after one barrier that ends the set-up (per-angle constants from the plan's
// FwdAngleRec table) they walk the same rows at nearly the same columns and
// share the L1 lines, and never wait on one another again.
// Bins 0 and nd-1 are recomputed by the warp whose strip holds them, with one
// lane per row deciding on the reference's own float s for the few pixels
// around those bins.
#include <climits>
#include <cmath>

#include "ctb_internal.h"

namespace ctb {
namespace {

constexpr int LANES = 32;
constexpr int PCH = kFwdRows;
constexpr int GMAX = kFwdGroup;
constexpr int THREADS = LANES * GMAX;
constexpr int NP = kFwdPlanes;          // float4 planes (4 slices each) per thread
constexpr float kRound = 12582912.0f;   // 1.5 * 2^23: x + kRound rounds x to an integer
constexpr int kRoundBits = 0x4B400000;  // bit pattern of kRound
static_assert(kFwdGuard >= 50, "the walked windows reach 50 columns outside the image (see strip_rows)");
static_assert(PCH == 16, "a chunk is two 8-row bands of the non-zero bounds");
static_assert(NP == 2, "a pixel holds the 8 slices of a plane pair: two float4, one 32-byte load");

struct FAngle {
    double q0;   // crossing of the strip's lower edge (bin b_lo = k K - 1) at p = 0
    double inv;  // dq*/db = 1 / kq
    double dq;   // dq*/dp = -kp / kq
    float dqf;
    float akq;     // |kq|: bins per pixel step along the walked row
    float cf, sf;  // the reference's float cos/sin
    int a;
    int p_lo, p_hi;  // rows where the strip meets the non-zero box and disc
    int c_lo, c_hi;  // columns of the non-zero box
    int neg;         // kq < 0: the strip's columns decrease with the bin
};

__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
// One pixel of a plane pair: 8 slices in 32 bytes (32-byte aligned), one load.
__device__ __forceinline__ void ld_pixel(const float4* p, float4 (&v)[NP]) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(v[0].x), "=f"(v[0].y), "=f"(v[0].z), "=f"(v[0].w), "=f"(v[1].x), "=f"(v[1].y), "=f"(v[1].z),
          "=f"(v[1].w)
        : "l"(p));
}
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }

// Lane l's first bin (relative to b_lo): floor((l - 1/2) |kq|). The combine
// step evaluates exactly this expression again for other lanes.
__device__ __forceinline__ int lane_bin(int l, float akq) {
    return static_cast<int>(floorf((static_cast<float>(l) - 0.5f) * akq));
}

// One chunk of the walk. Row pp crosses the strip's lower edge at column
// base + A, A = fa + pp dq (float); the lanes read columns cb + S l, cb =
// base + rint(A). With phi = S (rint(A) - A), lane l's pixel lies u = (l -
// phi) |kq| bins above the edge, and y = u - m_l - 1 = cl1 - phi |kq| (cl1 =
// l |kq| - m_l - 1) in [-1, 1] gives its hat weights for bins m_l, m_l + 1,
// m_l + 2: max(-y, 0), 1 - |y|, max(y, 0).
// Reads stay inside the zero border: a walked row lies within one row of the
// range where the strip's columns, at most 31.5 wide, come within kReach = 2
// columns of the non-zero box (or of the image without bounds), or at most 15
// rows beyond it (chunks start on multiples of 16), and |dq| <= 1. So the
// window start is at least 2 + 1 + 31.5 + 0.5 + 15 = 50 columns left of the
// box's first column and at most 2 + 1 + 0.5 + 15 = 18.5 right of its last
// (mirrored for S < 0), and the 32-column window stays within 50 columns of
// the image on either side: inside the kFwdGuard = 64 border, which reads as
// zeros.
// Rows P0 .. P0 + NR - 1 of the chunk.
template <int S, int P0, int NR>
__device__ __forceinline__ void strip_rows(const float4* __restrict__ rowp, int pitch, int base, float fa,
                                           float dqf, float akq, float cl1, int lane, float2 (&acc)[3][2 * NP]) {
#pragma unroll
    for (int pp = P0; pp < P0 + NR; ++pp) {
        const float A = fmaf(static_cast<float>(pp), dqf, fa);
        const float tr = A + kRound;
        const float rr = tr - kRound;
        const int cb = base + (__float_as_int(tr) - kRoundBits);
        const float y = fmaf(S > 0 ? rr - A : A - rr, akq, cl1);
        const float w0 = fmaxf(-y, 0.0f), w2 = fmaxf(y, 0.0f), w1 = 1.0f - fabsf(y);
        const float2 W0 = make_float2(w0, w0), W1 = make_float2(w1, w1), W2 = make_float2(w2, w2);
        const float4* px = rowp + 2 * (static_cast<long long>(pp) * pitch + cb + S * lane);
        float4 v[NP];
        ld_pixel(px, v);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            acc[0][2 * k] = __ffma2_rn(W0, lo2(v[k]), acc[0][2 * k]);
            acc[0][2 * k + 1] = __ffma2_rn(W0, hi2(v[k]), acc[0][2 * k + 1]);
            acc[1][2 * k] = __ffma2_rn(W1, lo2(v[k]), acc[1][2 * k]);
            acc[1][2 * k + 1] = __ffma2_rn(W1, hi2(v[k]), acc[1][2 * k + 1]);
            acc[2][2 * k] = __ffma2_rn(W2, lo2(v[k]), acc[2][2 * k]);
            acc[2][2 * k + 1] = __ffma2_rn(W2, hi2(v[k]), acc[2][2 * k + 1]);
        }
    }
}

// Bins 0 and nd-1 by the reference's rules (SerialBackend.cpp:109-120), on
// its own float s: bin 0 takes (1 - frac) v from the pixels with floor(s) =
// 0, bin nd-1 takes frac v from floor(s) = nd-2 and v from floor(s) = nd-1.
// Lane l takes rows r_lo + l, r_lo + l + 32, ... up to r_hi; in each row the
// candidates are the columns whose exact s lies within 1/64 of [lo, hi] =
// [0, 1] (bin 0) or [nd-2, nd] (bin nd-1), the reference's float s being
// much closer than that to the exact one. The lanes' sums are added by a
// fixed shuffle tree; every lane returns the total.
__device__ __noinline__ void edge_bin(const float4* __restrict__ plane, int pitch, int nq,
                                      const FAngle& f, int b_lo, int e, int nd, int r_lo, int r_hi, bool rows,
                                      float cxf, float cyf, int lane, float2 (&sum)[2 * NP]) {
#pragma unroll
    for (int j = 0; j < 2 * NP; ++j) sum[j] = make_float2(0.0f, 0.0f);
    const double lo = e == 0 ? 0.0 : nd - 2.0, hi = e == 0 ? 1.0 : static_cast<double>(nd);
    const double da = (lo - 1.0 / 64 - b_lo) * f.inv, db = (hi + 1.0 / 64 - b_lo) * f.inv;
    const float dcs = static_cast<float>(nd / 2);
    for (int p = r_lo + lane; p <= r_hi; p += LANES) {
        const double qp = fma(static_cast<double>(p), f.dq, f.q0);
        const int c0 = static_cast<int>(ceil(qp + fmin(da, db)));
        const int c1 = min(static_cast<int>(floor(qp + fmax(da, db))), c0 + 5);
        for (int c = max(c0, 0); c <= min(c1, nq - 1); ++c) {
            const float xg = static_cast<float>(rows ? c : p);
            const float yg = static_cast<float>(rows ? p : c);
            const float ss = __fadd_rn(__fadd_rn(__fmul_rn(__fsub_rn(xg, cxf), f.cf),
                                                 __fmul_rn(__fsub_rn(yg, cyf), f.sf)), dcs);
            const float fl = floorf(ss);
            const int i0 = static_cast<int>(fl);
            const float fr = __fsub_rn(ss, fl);
            float wgt = 0.0f;
            if (e == 0) wgt = i0 == 0 ? __fsub_rn(1.0f, fr) : 0.0f;
            else wgt = i0 == nd - 2 ? fr : (i0 == nd - 1 ? 1.0f : 0.0f);
            if (wgt == 0.0f) continue;
            const float2 W = make_float2(wgt, wgt);
            const float4* px = plane + 2 * (static_cast<long long>(p) * pitch + c);
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                const float4 v = __ldg(px + k);
                sum[2 * k] = __ffma2_rn(W, lo2(v), sum[2 * k]);
                sum[2 * k + 1] = __ffma2_rn(W, hi2(v), sum[2 * k + 1]);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 2 * NP; ++j)
        for (int o = 16; o > 0; o >>= 1) {
            sum[j].x += __shfl_xor_sync(0xffffffffu, sum[j].x, o);
            sum[j].y += __shfl_xor_sync(0xffffffffu, sum[j].y, o);
        }
}

__global__ void __launch_bounds__(THREADS, 7) k_forward(const float4* __restrict__ img,
                                                        const float4* __restrict__ imgT, int w,
                                                        int h, int nz, int na, int nd,
                                                        const int4* __restrict__ groups,
                                                        const FwdAngleRec* __restrict__ arec,
                                                        const int4* __restrict__ box,
                                                        const int2* __restrict__ band,
                                                        float* __restrict__ sino) {
    __shared__ FAngle fa[GMAX];
    __shared__ int erow[GMAX][4];                      // edge-pass rows: bin 0 [lo, hi], bin nd-1 [lo, hi]

    const int4 grp = groups[blockIdx.y];
    const int cnt = grp.y;
    const bool rows = grp.z == 0;
    const int K = grp.w;  // output bins per strip for this group
    if (blockIdx.x * K >= nd) return;  // the group has fewer strips than the grid (uniform per CTA)
    const int b_lo = blockIdx.x * K - 1;       // the strip's lower edge bin
    const int nout = min(K, nd - 1 - b_lo);    // output bins b_lo + 1 .. b_lo + nout
    const bool has0 = b_lo < 0, has_last = b_lo + nout == nd - 1;
    const int lane = threadIdx.x, ja = threadIdx.y;
    const int tid = ja * LANES + lane;

    const int np = rows ? h : w;  // walked axis
    const int nq = rows ? w : h;  // gathered axis
    const double cq = rows ? 0.5 * (w - 1) : 0.5 * (h - 1);
    const double cp = rows ? 0.5 * (h - 1) : 0.5 * (w - 1);
    const double dcf = static_cast<double>(nd / 2);
    constexpr double kReach = 2.0;  // margin of the row ranges (columns)

    // p range (within rows [rl, rh]) where crossings [qa, qb] (at p = 0) come
    // within reach of columns [cl, ch]; idq = 1 / dq (the margins of one row
    // and kReach columns absorb its rounding)
    auto prange = [&](double qa, double qb, double dq, double idq, int cl, int ch, int rl, int rh, int& lo,
                      int& hi) {
        lo = rl;
        hi = rh;
        if (dq != 0.0) {
            const double pa0 = (cl - kReach - qa) * idq, pb0 = (ch + kReach - qa) * idq;
            const double pa1 = (cl - kReach - qb) * idq, pb1 = (ch + kReach - qb) * idq;
            lo = max(rl, static_cast<int>(floor(fmin(fmin(pa0, pb0), fmin(pa1, pb1)))) - 1);
            hi = min(rh, static_cast<int>(ceil(fmax(fmax(pa0, pb0), fmax(pa1, pb1)))) + 1);
        } else if (fmax(qa, qb) < cl - kReach || fmin(qa, qb) > ch + kReach) {
            hi = -1;
        }
    };

    if (tid < cnt) {
        // the non-zero box of the CTA's slices (all its 4-slice groups), as
        // walked rows [rl, rh] and gathered columns [cl, ch]
        const int ng4 = (nz + 3) / 4;
        // without bounds: the whole image and a disc through its corners
        int4 bx = box ? box[2 * blockIdx.z * NP] : make_int4(0, w - 1, 0, h - 1);
        int r4 = box ? box[2 * blockIdx.z * NP + 1].x : (w - 1) * (w - 1) + (h - 1) * (h - 1);
        for (int k = 1; k < NP && box; ++k) {
            if (blockIdx.z * NP + k >= ng4) break;
            const int4 b2 = box[2 * (blockIdx.z * NP + k)];
            bx = make_int4(min(bx.x, b2.x), max(bx.y, b2.y), min(bx.z, b2.z), max(bx.w, b2.w));
            r4 = max(r4, box[2 * (blockIdx.z * NP + k) + 1].x);
        }
        const int rl = rows ? bx.z : bx.x, rh = rows ? bx.w : bx.y;
        const int cl = rows ? bx.x : bx.z, ch = rows ? bx.y : bx.w;
        const FwdAngleRec R = arec[grp.x + tid];
        const int a = R.a;
        const double kq = R.kq;
        const double kp = R.kp;
        // s(q, p) = (q - cq) kq + (p - cp) kp + dcf = b  <=>  q = q0(b) + p dq
        FAngle f;
        f.inv = R.inv;
        f.dq = -kp * f.inv;
        f.q0 = cq + (static_cast<double>(b_lo) - dcf + cp * kp) * f.inv;
        f.dqf = static_cast<float>(f.dq);
        f.akq = static_cast<float>(fabs(kq));
        f.neg = kq < 0.0 ? 1 : 0;
        f.cf = R.cf;
        f.sf = R.sf;
        f.a = a;
        f.c_lo = cl;
        f.c_hi = ch;
        f.p_lo = 0;
        f.p_hi = -1;
        int e0 = 0, e1 = -1, e2 = 0, e3 = -1;
        if (ch >= cl) {  // an empty box (all slices zero) leaves no rows
            // the strip's pixels have s in (b_lo, b_lo + K + 1)
            const double idq = R.idq;
            prange(f.q0, f.q0 + (K + 1) * f.inv, f.dq, idq, cl, ch, rl, rh, f.p_lo, f.p_hi);
            // Rows where the strip meets the disc: in the frame
            // u' = (q - cq) kq + (p - cp) kp, v = (p - cp) kq - (q - cq) kp the
            // strip is u' in [U0, U1], the disc u'^2 + v^2 <= rad^2, and p - cp
            // = u' kp + v kq. The rectangle u' in [max(U0, -rad), min(U1, rad)],
            // |v| <= sqrt(rad^2 - m^2) (m the smallest |u'| there) holds their
            // intersection.
            // (single-precision roots: their error, ~1e-4 pixels, is far inside
            // the margins of 1.5 pixels and 2 rows)
            const double rad = 0.5 * sqrtf(static_cast<float>(r4)) + 1.5;
            const double u0 = static_cast<double>(b_lo) - dcf, u1 = u0 + K + 1;
            const double a0 = fmax(fmin(u0, u1), -rad), a1 = fmin(fmax(u0, u1), rad);
            if (a0 > a1) {
                f.p_hi = -1;
            } else {
                const double m = (a0 <= 0.0 && a1 >= 0.0) ? 0.0 : fmin(fabs(a0), fabs(a1));
                const double vm = sqrtf(static_cast<float>(fmax(0.0, rad * rad - m * m)));
                const double e0d = a0 * kp, e1d = a1 * kp, ev = vm * fabs(kq);
                const int dlo = static_cast<int>(floor(cp + fmin(e0d, e1d) - ev)) - 2;
                const int dhi = static_cast<int>(ceil(cp + fmax(e0d, e1d) + ev)) + 2;
                f.p_lo = max(f.p_lo, dlo);
                f.p_hi = min(f.p_hi, dhi);
            }
            // rows of the edge passes: s within [-1, 2] of bin 0, [nd-3, nd+1] of bin nd-1
            if (has0)
                prange(f.q0 + (-1 - b_lo) * f.inv, f.q0 + (2 - b_lo) * f.inv, f.dq, idq, cl, ch, rl, rh, e0, e1);
            if (has_last)
                prange(f.q0 + (nd - 3 - b_lo) * f.inv, f.q0 + (nd + 1 - b_lo) * f.inv, f.dq, idq, cl, ch, rl, rh, e2,
                       e3);
        }
        fa[tid] = f;
        erow[tid][0] = e0;
        erow[tid][1] = e1;
        erow[tid][2] = e2;
        erow[tid][3] = e3;
    }
    __syncthreads();
    const bool has_a = ja < cnt;
    const int ng4 = (nz + 3) / 4;    // float4 planes
    const int g0 = blockIdx.z * NP;  // first plane of the CTA
    bool any = false;
    for (int k = 0; k < cnt; ++k) any = any || fa[k].p_hi >= fa[k].p_lo;
    if (!any) {  // the strip meets no non-zero pixel at any angle of the group
        if (has_a && lane < nout)
            for (int z = 4 * g0; z < min(nz, 4 * (g0 + NP)); ++z)
                sino[(static_cast<long long>(z) * na + fa[ja].a) * nd + b_lo + 1 + lane] = 0.0f;
        return;
    }

    const int pitch = nq + 2 * kFwdGuard;
    // the CTA's plane pair: (np + PCH) rows of pitch pixels of 8 slices (two
    // float4). Pairs are allocated whole: a half past the last slice is read
    // but its sums are not stored
    const long long pstride = 2LL * (np + PCH) * pitch;
    const float4* plane = (rows ? img : imgT) + blockIdx.z * pstride + 2 * kFwdGuard;
    // 8-row bands of the walked axis: row bands (x ranges) of the group when
    // walking rows, its column bands (y ranges) when walking columns
    const int nby = (h + 7) / 8, nbx = (w + 7) / 8;
    const int nb_all = nby + nbx, nb_off = rows ? 0 : nby, nb_p = rows ? nby : nbx;

    float2 acc[3][2 * NP];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int j = 0; j < 2 * NP; ++j) acc[r][j] = make_float2(0.0f, 0.0f);
    if (has_a) {
        const FAngle& f = fa[ja];
        const float akq = f.akq;
        const int ml = lane_bin(lane, akq);
        const float cl1 = fmaf(static_cast<float>(lane), akq, -static_cast<float>(ml + 1));
        // chunks start on multiples of PCH, so that warps whose row ranges
        // overlap walk the same rows at about the same time; each half of a
        // chunk is then exactly one 8-row band
        for (int p0 = f.p_lo & ~(PCH - 1); p0 <= f.p_hi; p0 += PCH) {
            const double qs = fma(static_cast<double>(p0), f.dq, f.q0);
            const double qfl = floor(qs);
            const int base = static_cast<int>(qfl);
            const float fq = static_cast<float>(qs - qfl);
            // Each half walks only when the columns its lanes read, base +
            // rint(fq + pp dqf) + S l with fq in [0, 1), meet its non-zero
            // columns: the range of its band over the CTA's slice groups
            // (none for rows past the image), or the box without bands. A
            // skipped half adds only zeros.
            bool walk[2];
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
                int cl = f.c_lo, ch = f.c_hi;
                if (band) {
                    cl = INT_MAX;
                    ch = -1;
                    const int bi = (p0 >> 3) + hh;
                    for (int k = 0; k < NP && bi < nb_p; ++k) {
                        if (g0 + k >= ng4) break;
                        const int2 r = __ldg(band + static_cast<long long>(g0 + k) * nb_all + nb_off + bi);
                        cl = min(cl, r.x);
                        ch = max(ch, r.y);
                    }
                }
                const float e0 = static_cast<float>(8 * hh) * f.dqf, e1 = static_cast<float>(8 * hh + 7) * f.dqf;
                const int lo = base + static_cast<int>(floorf(fminf(e0, e1))) - 1 - (f.neg ? LANES - 1 : 0);
                const int hi = base + static_cast<int>(ceilf(fmaxf(e0, e1))) + 2 + (f.neg ? 0 : LANES - 1);
                walk[hh] = ch >= cl && hi >= cl && lo <= ch;
            }
            const bool w0 = walk[0], w1 = walk[1];
            const float4* rowp = plane + 2LL * p0 * pitch;
            if (f.neg) {
                if (w0) strip_rows<-1, 0, 8>(rowp, pitch, base, fq, f.dqf, akq, cl1, lane, acc);
                if (w1) strip_rows<-1, 8, 8>(rowp, pitch, base, fq, f.dqf, akq, cl1, lane, acc);
            } else {
                if (w0) strip_rows<1, 0, 8>(rowp, pitch, base, fq, f.dqf, akq, cl1, lane, acc);
                if (w1) strip_rows<1, 8, 8>(rowp, pitch, base, fq, f.dqf, akq, cl1, lane, acc);
            }
        }
    }
    if (!has_a) return;
    const FAngle& f = fa[ja];
    const long long zst = static_cast<long long>(na) * nd;  // slice stride of the sinograms
    const long long ob = static_cast<long long>(f.a) * nd;
    // Output bin t = lane + 1 of the strip is the sum, in lane order, of
    // accumulator t - m_l of every lane l with m_l in [t - 2, t]. Lanes with
    // equal m_l form runs of one or two (m_l + 2 - m_l >= 2|kq| > 1) and the
    // runs' values are -1, 0, 1, ... in lane order (consecutive m differ by at
    // most |kq| <= 1, and m_0 = -1), so run m starts at the (m + 1)-th set bit
    // (counting from 0) of `firsts`. The terms come by warp shuffles.
    constexpr unsigned kAll = 0xffffffffu;
    const int ml = lane_bin(lane, f.akq);
    const int mprev = __shfl_up_sync(kAll, ml, 1);
    const unsigned firsts = __ballot_sync(kAll, lane == 0 || mprev != ml);
    const int t = lane + 1;
    float2 sum[2 * NP];
#pragma unroll
    for (int j = 0; j < 2 * NP; ++j) sum[j] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int r = 2; r >= 0; --r) {
        const unsigned l0 = __fns(firsts, 0, t - r + 2);  // first lane of run t - r (or ~0u: none)
        const bool ok0 = l0 < LANES;
        const bool ok1 = ok0 && l0 + 1 < LANES && !((firsts >> (l0 + 1)) & 1u);
        const int s0 = ok0 ? static_cast<int>(l0) : lane, s1 = ok1 ? static_cast<int>(l0) + 1 : lane;
#pragma unroll
        for (int j = 0; j < 2 * NP; ++j) {
            const float2 a0 = make_float2(__shfl_sync(kAll, acc[r][j].x, s0), __shfl_sync(kAll, acc[r][j].y, s0));
            const float2 a1 = make_float2(__shfl_sync(kAll, acc[r][j].x, s1), __shfl_sync(kAll, acc[r][j].y, s1));
            if (ok0) sum[j] = __fadd2_rn(sum[j], a0);
            if (ok1) sum[j] = __fadd2_rn(sum[j], a1);
        }
    }
    const int b = b_lo + t;
    if (lane < nout && b != 0 && b != nd - 1) {
#pragma unroll
        for (int j = 0; j < 2 * NP; ++j) {
            const int z = 4 * g0 + 2 * j;  // slices z, z + 1 of pair j
            if (z < nz) sino[z * zst + ob + b] = sum[j].x;
            if (z + 1 < nz) sino[(z + 1) * zst + ob + b] = sum[j].y;
        }
    }
    // bins 0 and nd-1 on the reference's own rules
    const float cxf = static_cast<float>(w - 1) * 0.5f, cyf = static_cast<float>(h - 1) * 0.5f;
    for (int side = 0; side < 2; ++side) {
        if (!(side == 0 ? has0 : has_last)) continue;
        const int eb = side == 0 ? 0 : nd - 1;
        float2 sum[2 * NP];
        edge_bin(plane, pitch, nq, f, b_lo, eb, nd, erow[ja][2 * side], erow[ja][2 * side + 1], rows, cxf,
                 cyf, lane, sum);
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < 2 * NP; ++j) {
                const int z = 4 * g0 + 2 * j;
                if (z < nz) sino[z * zst + ob + eb] = sum[j].x;
                if (z + 1 < nz) sino[(z + 1) * zst + ob + eb] = sum[j].y;
            }
        }
    }
}

// One thread per angle group: the per-angle constants of its angles (the
// expressions the projector's set-up evaluated itself before).
__global__ void k_fwd_angles(const int4* __restrict__ groups, int ngroups, const int* __restrict__ order,
                             Trig trig, FwdAngleRec* __restrict__ rec) {
    const int gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= ngroups) return;
    const int4 grp = groups[gi];
    const bool rows = grp.z == 0;
    for (int k = 0; k < grp.y; ++k) {
        const int a = order[grp.x + k];
        const double2 tc = trig.cs[a];
        FwdAngleRec r;
        r.kq = rows ? tc.x : tc.y;
        r.kp = rows ? tc.y : tc.x;
        r.inv = 1.0 / r.kq;
        const double dq = -r.kp * r.inv;
        r.idq = dq != 0.0 ? 1.0 / dq : 0.0;
        const float2 tf = trig.csf[a];
        r.cf = tf.x;
        r.sf = tf.y;
        r.a = a;
        r.pad = 0;
        rec[grp.x + k] = r;
    }
}

}  // namespace

cudaError_t launch_forward(const float4* d_img, const float4* d_imgT, int w, int h, int nz,
                           int na, int nd, const int4* d_groups, int ngroups, int max_strips,
                           const FwdAngleRec* d_rec, const int4* d_box, const int2* d_band, float* d_sino,
                           cudaStream_t st) {
    const dim3 grid(max_strips, ngroups, ((nz + 3) / 4 + NP - 1) / NP);
    k_forward<<<grid, dim3(LANES, GMAX), 0, st>>>(d_img, d_imgT, w, h, nz, na, nd, d_groups, d_rec, d_box,
                                                  d_band, d_sino);
    return cudaGetLastError();
}

cudaError_t launch_fwd_angles(const int4* d_groups, int ngroups, const int* d_order, Trig trig,
                              FwdAngleRec* d_rec, cudaStream_t st) {
    k_fwd_angles<<<(ngroups + 127) / 128, 128, 0, st>>>(d_groups, ngroups, d_order, trig, d_rec);
    return cudaGetLastError();
}

}  // namespace ctb
