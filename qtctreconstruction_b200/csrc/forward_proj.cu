// forward_proj.cu — the forward projector (the RadonTransform stage of the
// FBP path).
//
// The reference's forward projector (SerialBackend::computeSinogram,
// SerialBackend.cpp:59-136) splats every non-zero pixel onto the two detector
// bins around s = (x-cx)cos + (y-cy)sin + floor(nd/2) with weights
// (1 - frac, frac), frac = s - floor(s). Here the splat is reorganised by
// detector interval: a thread owns interval j (the pixels with floor(s) = j)
// of one angle and walks it through the image, reading each of its pixels
// once and keeping two sums, so that every pixel is read once per angle and
// its two contributions stay in registers; bin j + 1 is then the frac part of
// interval j plus the (1 - frac) part of interval j + 1, combined across
// neighbouring threads at the end. Sinogram stores are coalesced by bin.
//
// The interval family is walked along the image axis it is closest to (rows
// when |cos| >= |sin|, else columns of the transposed copy), so an interval
// holds one or two pixels of each walked row. Its two boundaries (the
// crossings of bins j and j+1) are evaluated in double once per chunk of
// PCH = 16 rows as an integer column plus a float offset, and stepped in float
// within the chunk; threads that share a boundary evaluate it identically, so
// membership (an exact comparison of a pixel column with a boundary) gives a
// partition of the pixels. The two edge intervals (0 and nd-1), where the
// reference's rules are discontinuous, decide membership on the reference's
// own float s (SerialBackend.cpp:109-120) on a separate, warp-uniform path.
//
// A CTA is one warp per angle of a group of up to GMAX = 4 angles that share
// the walked axis; lane x of every warp owns interval jb + x of FB = 32
// consecutive intervals (FB - 1 output bins, the last interval only feeds the
// neighbour sum), for 4 NP slices (NP float4 planes of the normalised image).
// Pixels are read straight from the zero-bordered planes through L1: the
// warps of a CTA walk nearly the same rows at the same time and share the
// lines. Warps never wait on one another, and the CTA's warps have nearly
// equal row counts, so CTAs retire evenly. Accumulation runs on packed FP32x2
// instructions.
#include <climits>
#include <cmath>

#include "ctb_internal.h"

namespace ctb {
namespace {

constexpr int FB = kFwdRays;  // intervals per CTA (one warp per angle)
constexpr int OUT = FB - 1;   // output bins per CTA
static_assert(FB == 32, "a warp owns the CTA's intervals of one angle");
constexpr int PCH = kFwdRows;
constexpr int GMAX = kFwdGroup;
constexpr int AY = GMAX;  // angle lanes per CTA
constexpr int THREADS = FB * AY;
constexpr int NP = kFwdPlanes;  // float4 planes (4 slices each) per thread
constexpr float kRound = 12582912.0f;   // 1.5 * 2^23: x + kRound rounds x to an integer
constexpr int kRoundBits = 0x4B400000;  // bit pattern of kRound

struct FAngle {
    double q0;   // crossing q*(jb, p = 0) of the CTA's first interval boundary
    double inv;  // dq*/db = 1 / kq
    double dq;   // dq*/dp = -kp / kq
    float dqf;
    float akq;     // |kq|: fraction per pixel step inside an interval
    float cf, sf;  // the reference's float cos/sin
    int a;
    int p_lo, p_hi;  // rows where an interval of the CTA meets the non-zero box
    int c_lo, c_hi;  // columns of the non-zero box
    int edge;        // interval 0 or nd-1 of this CTA meets the box at this angle
    int neg;   // kq < 0: crossings decrease with the bin
};

// Interval boundary t (the crossing of bin jb + t) at a chunk's first row p0,
// as the integer column floor(q*) and the float offset q* - floor(q*); row pp
// of the chunk crosses at base + (f + pp dq). Every thread that needs
// boundary t evaluates exactly this expression on the same operands, so the
// two threads sharing a boundary hold the same integer and the same floats.
// The float stays below |dq| (PCH - 1) + 1, where its rounding is ~16x finer
// than that of a float column coordinate.
struct Bound {
    int base;
    float f;
};
__device__ __forceinline__ Bound boundary(const FAngle& f, int t, int p0) {
    const double qstar = fma(static_cast<double>(p0), f.dq, fma(static_cast<double>(t), f.inv, f.q0));
    const double qfl = floor(qstar);
    return Bound{static_cast<int>(qfl), static_cast<float>(qstar - qfl)};
}

// A chunk is skipped exactly when both boundaries lie left of column
// c_lo - 2, or right of column c_hi + 1, at its first and last rows, [c_lo,
// c_hi] being the columns of the non-zero box (inside the image): the
// boundaries are linear in the row, so the interval (at most sqrt 2 wide) then
// holds only zero pixels at every row of the chunk. Otherwise some boundary is
// within two columns of the image at some row; moving at most one column per
// row, every candidate column of the chunk stays within kFwdRows + 5 columns
// of the image, inside the zero border (kFwdGuard = kFwdRows + 8).
__device__ __forceinline__ bool chunk_meets_box(const Bound& ba, const Bound& bb, float dqf, int c_lo,
                                                int c_hi) {
    const float e = (PCH - 1) * dqf;
    const float a0 = static_cast<float>(ba.base) + ba.f, b0 = static_cast<float>(bb.base) + bb.f;
    const float lo = fminf(fminf(a0, a0 + e), fminf(b0, b0 + e));
    const float hi = fmaxf(fmaxf(a0, a0 + e), fmaxf(b0, b0 + e));
    return hi >= static_cast<float>(c_lo - 2) && lo <= static_cast<float>(c_hi + 1);
}

__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }

// The fast path over one chunk. Interval j holds the pixels q of a row with
// floor(s(q)) = j: q in [A, B) for kq > 0, q in (B, A] for kq < 0, A and B the
// crossings of bins j and j+1. Its width is R = 1/|kq| in [1, sqrt 2], so with
// rr = rint(A - baseA) the members are among baseA + rr and baseA + rr + S
// (S the walking direction), decided by exact comparisons with A and B. A
// member at distance d = |q - A| has frac = d |kq|: it adds (1 - frac) v to
// bin j and frac v to bin j + 1. The thread keeps sum(v) and sum(d v); |kq|
// is applied once at the end. A non-member skips its load (predicated off,
// so it costs no L1 wavefront) and its register's stale finite value enters
// with weight 0.
template <int S>
__device__ __forceinline__ void splat_rows(const float4* __restrict__ rowp, long long pofs, int pitch,
                                           Bound ba, Bound bb, float dqf, float2 (&sv)[2 * NP],
                                           float2 (&sd)[2 * NP]) {
    // pixel baseA + r + S lies before B iff r + cab < fB (S > 0), > fB (S < 0)
    const float cab = static_cast<float>(ba.base - bb.base + S);
    float4 pv0[NP], pv1[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) pv0[k] = pv1[k] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int pp = 0; pp < PCH; ++pp) {
        const float A = fmaf(static_cast<float>(pp), dqf, ba.f);
        const float B = fmaf(static_cast<float>(pp), dqf, bb.f);
        const float tr = A + kRound;
        const float rr = tr - kRound;
        const int ia = __float_as_int(tr) - kRoundBits + ba.base + pp * pitch;
        const float x1 = rr + cab;
        const bool m0 = S > 0 ? rr >= A : rr <= A;
        const bool m1 = S > 0 ? x1 < B : x1 > B;
        const float d0 = S > 0 ? rr - A : A - rr;
        const float c0f = m0 ? 1.0f : 0.0f, c1f = m1 ? 1.0f : 0.0f;
        const float2 c0 = make_float2(c0f, c0f), c1 = make_float2(c1f, c1f);
        const float2 u0 = make_float2(m0 ? d0 : 0.0f, m0 ? d0 : 0.0f);
        const float2 u1 = make_float2(m1 ? d0 + 1.0f : 0.0f, m1 ? d0 + 1.0f : 0.0f);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            if (m0) pv0[k] = __ldg(rowp + k * pofs + ia);
            if (m1) pv1[k] = __ldg(rowp + k * pofs + ia + S);
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const float4 v0 = pv0[k], v1 = pv1[k];
            sv[2 * k] = __ffma2_rn(c1, lo2(v1), __ffma2_rn(c0, lo2(v0), sv[2 * k]));
            sv[2 * k + 1] = __ffma2_rn(c1, hi2(v1), __ffma2_rn(c0, hi2(v0), sv[2 * k + 1]));
            sd[2 * k] = __ffma2_rn(u1, lo2(v1), __ffma2_rn(u0, lo2(v0), sd[2 * k]));
            sd[2 * k + 1] = __ffma2_rn(u1, hi2(v1), __ffma2_rn(u0, hi2(v0), sd[2 * k + 1]));
        }
    }
}

// The edge intervals: SerialBackend.cpp:109-120 decides on its own float s
// which pixels count at the two discontinuities of its rules: a pixel reaches
// bin 0 only from floor(s) == 0 (interval -1 adds nothing), and bin nd-1 takes
// the full value from floor(s) == nd-1 and nothing from floor(s) >= nd. So
// interval 0 takes its lower side from the reference's s >= 0 and interval
// nd-1 its upper side from s < nd (with weight 1 on bin nd-1, recorded as
// d = 0); every other side is the exact comparison of the fast path. Four
// candidates around rint(A) cover the reference's float rounding.
struct Sums {
    float2 v[2 * NP], d[2 * NP];
};
__device__ __noinline__ Sums splat_rows_edge(const float4* __restrict__ rowp, long long pofs, int pitch,
                                             const FAngle& f, Bound ba, Bound bb, int p0, int j, int nd,
                                             bool rows, float cxf, float cyf, Sums acc) {
    const int S = f.neg ? -1 : 1;
    const float cab = static_cast<float>(ba.base - bb.base);
    const float dcs = static_cast<float>(nd / 2);
    for (int pp = 0; pp < PCH; ++pp) {
        const float A = fmaf(static_cast<float>(pp), f.dqf, ba.f);
        const float B = fmaf(static_cast<float>(pp), f.dqf, bb.f);
        const float rr = rintf(A);
        for (int k = -1; k <= 2; ++k) {
            const float r = rr + static_cast<float>(S * k);  // pixel column baseA + r
            const int qg = ba.base + static_cast<int>(r);
            const int pg = p0 + pp;
            const float xg = static_cast<float>(rows ? qg : pg);
            const float yg = static_cast<float>(rows ? pg : qg);
            const float ss = __fadd_rn(__fadd_rn(__fmul_rn(__fsub_rn(xg, cxf), f.cf),
                                                 __fmul_rn(__fsub_rn(yg, cyf), f.sf)), dcs);
            const float x = r + cab;  // the pixel relative to baseB
            const bool lower = j == 0 ? ss >= 0.0f : (S > 0 ? r >= A : r <= A);
            const bool upper = j == nd - 1 ? ss < static_cast<float>(nd) : (S > 0 ? x < B : x > B);
            if (!(lower && upper)) continue;
            const float d = j == nd - 1 ? 0.0f : fmaxf(0.0f, S > 0 ? r - A : A - r);
            const float2 w = make_float2(d, d);
            for (int pl = 0; pl < NP; ++pl) {
                const float4 v = __ldg(rowp + pl * pofs + pp * pitch + qg);
                acc.v[2 * pl] = __fadd2_rn(acc.v[2 * pl], lo2(v));
                acc.v[2 * pl + 1] = __fadd2_rn(acc.v[2 * pl + 1], hi2(v));
                acc.d[2 * pl] = __ffma2_rn(w, lo2(v), acc.d[2 * pl]);
                acc.d[2 * pl + 1] = __ffma2_rn(w, hi2(v), acc.d[2 * pl + 1]);
            }
        }
    }
    return acc;
}

__global__ void __launch_bounds__(THREADS, 7) k_forward(const float4* __restrict__ img,
                                                        const float4* __restrict__ imgT, int w,
                                                        int h, int nz, int na, int nd, Trig trig,
                                                        const int4* __restrict__ groups,
                                                        const int* __restrict__ order,
                                                        const int4* __restrict__ box,
                                                        const int2* __restrict__ band,
                                                        float* __restrict__ sino) {
    __shared__ FAngle fa[GMAX];

    const int ob0 = blockIdx.x * OUT;  // first output bin of the CTA
    const int nout = min(OUT, nd - ob0);
    const int jb = ob0 - 1;     // interval of thread x: jb + x, boundaries t = x, x + 1
    const int tmax = nout + 1;  // last boundary of the CTA
    const int4 grp = groups[blockIdx.y];
    const int cnt = grp.y;
    const bool rows = grp.z == 0;
    const int tx = threadIdx.x, ty = threadIdx.y;  // tx: lane (interval), ty: warp (angle)
    const int tid = ty * FB + tx;
    const int j = jb + tx;

    const int np = rows ? h : w;  // walked axis
    const int nq = rows ? w : h;  // gathered axis
    const double cq = rows ? 0.5 * (w - 1) : 0.5 * (h - 1);
    const double cp = rows ? 0.5 * (h - 1) : 0.5 * (w - 1);
    const double dcf = static_cast<double>(nd / 2);
    constexpr double kReach = 2.0;  // an interval is at most sqrt 2 wide

    // p range (within rows [rl, rh]) where crossings [qa, qb] (at p = 0) come
    // within reach of columns [cl, ch]
    auto prange = [&](double qa, double qb, double dq, int cl, int ch, int rl, int rh, int& lo, int& hi) {
        lo = rl;
        hi = rh;
        if (dq != 0.0) {
            const double pa0 = (cl - kReach - qa) / dq, pb0 = (ch + kReach - qa) / dq;
            const double pa1 = (cl - kReach - qb) / dq, pb1 = (ch + kReach - qb) / dq;
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
        // every non-zero pixel lies within rad of the image centre
        const int a = order[grp.x + tid];
        const double2 tc = trig.cs[a];
        const double kq = rows ? tc.x : tc.y;
        const double kp = rows ? tc.y : tc.x;
        // s(q, p) = (q - cq) kq + (p - cp) kp + dcf = b  <=>  q = q0(b) + p dq
        FAngle f;
        f.inv = 1.0 / kq;
        f.dq = -kp * f.inv;
        f.q0 = cq + (static_cast<double>(jb) - dcf + cp * kp) * f.inv;
        f.dqf = static_cast<float>(f.dq);
        f.akq = static_cast<float>(fabs(kq));
        f.neg = kq < 0.0 ? 1 : 0;
        const float2 tf = trig.csf[a];
        f.cf = tf.x;
        f.sf = tf.y;
        f.a = a;
        f.c_lo = cl;
        f.c_hi = ch;
        f.p_lo = 0;
        f.p_hi = -1;
        f.edge = 0;
        if (ch >= cl) {  // an empty box (all slices zero) leaves no rows
            prange(f.q0, f.q0 + tmax * f.inv, f.dq, cl, ch, rl, rh, f.p_lo, f.p_hi);
            // Rows where the intervals' strip meets the disc: in the frame
            // u' = (q - cq) kq + (p - cp) kp, v = (p - cp) kq - (q - cq) kp the
            // strip is u' in [U0, U1] (boundaries t = 0 and tmax), the disc
            // u'^2 + v^2 <= rad^2, and p - cp = u' kp + v kq. The rectangle
            // u' in [max(U0, -rad), min(U1, rad)], |v| <= sqrt(rad^2 - m^2)
            // (m the smallest |u'| there) holds their intersection.
            const double rad = 0.5 * sqrt(static_cast<double>(r4)) + 1.5;
            const double u0 = static_cast<double>(jb) - dcf, u1 = u0 + tmax;
            const double a0 = fmax(fmin(u0, u1), -rad), a1 = fmin(fmax(u0, u1), rad);
            if (a0 > a1) {
                f.p_hi = -1;
            } else {
                const double m = (a0 <= 0.0 && a1 >= 0.0) ? 0.0 : fmin(fabs(a0), fabs(a1));
                const double vm = sqrt(fmax(0.0, rad * rad - m * m));
                const double e0 = a0 * kp, e1 = a1 * kp, ev = vm * fabs(kq);
                const int dlo = static_cast<int>(floor(cp + fmin(e0, e1) - ev)) - 2;
                const int dhi = static_cast<int>(ceil(cp + fmax(e0, e1) + ev)) + 2;
                f.p_lo = max(f.p_lo, dlo);
                f.p_hi = min(f.p_hi, dhi);
            }
            for (int ej : {0, nd - 1}) {
                const int et = ej - jb;  // thread of the edge interval
                if (et < 0 || et > nout) continue;
                int lo, hi;
                prange(f.q0 + et * f.inv, f.q0 + (et + 1) * f.inv, f.dq, cl, ch, rl, rh, lo, hi);
                if (hi >= lo) f.edge = 1;
            }
        }
        fa[tid] = f;
    }
    __syncthreads();
    const int ja = ty;  // this thread's angle of the group
    const bool has_a = ja < cnt;
    const bool outs = tx < nout && has_a;  // thread writes output bin ob0 + tx
    const int ng4 = (nz + 3) / 4;          // float4 planes
    const int g0 = blockIdx.z * NP;        // first plane of the CTA
    bool any = false;
    for (int k = 0; k < cnt; ++k) any = any || fa[k].p_hi >= fa[k].p_lo;
    if (!any) {  // no interval of this CTA meets the image
        if (outs)
            for (int z = 4 * g0; z < min(nz, 4 * (g0 + NP)); ++z)
                sino[(static_cast<long long>(z) * na + fa[ja].a) * nd + ob0 + tx] = 0.0f;
        return;
    }

    const int pitch = nq + 2 * kFwdGuard;
    const long long pstride = static_cast<long long>(np + PCH) * pitch;
    const float4* plane = (rows ? img : imgT) + g0 * pstride + kFwdGuard;
    // a missing last plane of an odd plane count re-reads the first (not stored)
    const long long pofs = g0 + 1 < ng4 ? pstride : 0;

    // rows this warp's intervals can touch at its angle (warp-uniform)
    const int wlo = has_a ? fa[ja].p_lo : 0, whi = has_a ? fa[ja].p_hi : -1;
    // interval -1 adds nothing (the reference drops floor(s) < 0); threads
    // past the CTA's last interval idle
    const bool live = has_a && tx <= nout && j >= 0;
    // a warp holding interval 0 or nd-1 at an angle where it meets the image
    // takes the reference-decision path
    const bool edge_a = has_a && fa[ja].edge;
    const bool neg = has_a && fa[ja].neg;
    const float cxf = static_cast<float>(w - 1) * 0.5f, cyf = static_cast<float>(h - 1) * 0.5f;

    // 8-row bands of the walked axis: row bands (x ranges) of the group when
    // walking rows, its column bands (y ranges) when walking columns
    const int nby = (h + 7) / 8, nbx = (w + 7) / 8;
    const int nb_all = nby + nbx, nb_off = rows ? 0 : nby, nb_p = rows ? nby : nbx;

    Sums acc;
#pragma unroll
    for (int k = 0; k < 2 * NP; ++k) acc.v[k] = acc.d[k] = make_float2(0.f, 0.f);
    if (live) {
        const FAngle& f = fa[ja];
        for (int p0 = wlo; p0 <= whi; p0 += PCH) {
            const Bound ba = boundary(f, tx, p0);
            const Bound bb = boundary(f, tx + 1, p0);
            // the chunk's columns: the non-zero ranges of the 8-row bands its
            // rows fall in, over the CTA's slice groups
            int cl = f.c_lo, ch = f.c_hi;
            if (band) {
                cl = INT_MAX;
                ch = -1;
                const int b1 = min((p0 + PCH - 1) >> 3, nb_p - 1);
                for (int k = 0; k < NP; ++k) {
                    if (blockIdx.z * NP + k >= ng4) break;
                    const int2* bk = band + static_cast<long long>(blockIdx.z * NP + k) * nb_all + nb_off;
                    for (int bi = p0 >> 3; bi <= b1; ++bi) {
                        const int2 r = __ldg(bk + bi);
                        cl = min(cl, r.x);
                        ch = max(ch, r.y);
                    }
                }
            }
            if (ch < cl || !chunk_meets_box(ba, bb, f.dqf, cl, ch)) continue;
            const float4* rowp = plane + static_cast<long long>(p0) * pitch;
            if (edge_a) acc = splat_rows_edge(rowp, pofs, pitch, f, ba, bb, p0, j, nd, rows, cxf, cyf, acc);
            else if (neg) splat_rows<-1>(rowp, pofs, pitch, ba, bb, f.dqf, acc.v, acc.d);
            else splat_rows<1>(rowp, pofs, pitch, ba, bb, f.dqf, acc.v, acc.d);
        }
    }
    // bin jb + x + 1 = frac part of interval x + (1 - frac) part of interval x + 1
    const float akq = has_a ? fa[ja].akq : 0.0f;
    const float2 ak = make_float2(akq, akq);
    float2 right[2 * NP], nxt[2 * NP];
#pragma unroll
    for (int k = 0; k < 2 * NP; ++k) {
        right[k] = __fmul2_rn(ak, acc.d[k]);
        const float2 left = make_float2(acc.v[k].x - right[k].x, acc.v[k].y - right[k].y);
        nxt[k].x = __shfl_down_sync(0xffffffffu, left.x, 1);
        nxt[k].y = __shfl_down_sync(0xffffffffu, left.y, 1);
    }
    if (!outs) return;
    const long long ob = static_cast<long long>(fa[ja].a) * nd + ob0 + tx;
#pragma unroll
    for (int k = 0; k < 2 * NP; ++k) {
        const int z = 4 * g0 + 2 * k;  // slices z, z + 1 of pair k
        if (z < nz) sino[static_cast<long long>(z) * na * nd + ob] = right[k].x + nxt[k].x;
        if (z + 1 < nz) sino[static_cast<long long>(z + 1) * na * nd + ob] = right[k].y + nxt[k].y;
    }
}

}  // namespace

cudaError_t launch_forward(const float4* d_img, const float4* d_imgT, int w, int h, int nz,
                           int na, int nd, Trig trig, const int4* d_groups, int ngroups,
                           const int* d_order, const int4* d_box, const int2* d_band, float* d_sino,
                           cudaStream_t st) {
    const dim3 grid((nd + OUT - 1) / OUT, ngroups, ((nz + 3) / 4 + NP - 1) / NP);
    k_forward<<<grid, dim3(FB, AY), 0, st>>>(d_img, d_imgT, w, h, nz, na, nd, trig, d_groups, d_order,
                                             d_box, d_band, d_sino);
    return cudaGetLastError();
}

}  // namespace ctb
