// forward.cu — preparation kernels of the forward projection: angle tables,
// per-slice statistics and the normalised, slice-interleaved image copies the
// projector reads (forward_proj.cu holds the projector itself).
#include <cfloat>
#include <climits>
#include <cmath>

#include "ctb_internal.h"

namespace ctb {
namespace {

// ------------------------------------------------------------------ trig
// cos/sin of the angle in double precision: theta/pi = deg/180 exactly
// representable as a double quotient; sincospi avoids the pi rounding.
__global__ void k_trig(const float* __restrict__ deg, int na, double2* __restrict__ cs) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    double s, c;
    sincospi(static_cast<double>(deg[a]) / 180.0, &s, &c);
    cs[a] = make_double2(c, s);
}

// ------------------------------------------------------------ slice stats
// stats[z] = {min, max, span_fwd, span_denorm} (SerialBackend.cpp:70-80, 298-300).
// With box set, also empties the non-zero bounding box of each 4-slice group
// that k_normalize then fills.
__global__ void __launch_bounds__(1024) k_slice_stats(const float* __restrict__ vol, long long npx,
                                                      float4* __restrict__ stats, int4* __restrict__ box,
                                                      int2* __restrict__ band, int nband) {
    const int z = blockIdx.x;
    if (box && threadIdx.x == 0 && (z & 3) == 0) {
        box[2 * (z >> 2)] = make_int4(INT_MAX, -1, INT_MAX, -1);
        box[2 * (z >> 2) + 1] = make_int4(-1, 0, 0, 0);
    }
    if (band && (z & 3) == 0)
        for (int i = threadIdx.x; i < nband; i += blockDim.x)
            band[static_cast<long long>(z >> 2) * nband + i] = make_int2(INT_MAX, -1);
    const float* p = vol + static_cast<long long>(z) * npx;
    float lo = FLT_MAX, hi = -FLT_MAX;
    if ((npx & 3) == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
        const float4* p4 = reinterpret_cast<const float4*>(p);
        for (long long i = threadIdx.x; i < npx / 4; i += blockDim.x) {
            const float4 v = __ldg(p4 + i);
            lo = fminf(lo, fminf(fminf(v.x, v.y), fminf(v.z, v.w)));
            hi = fmaxf(hi, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
        }
    } else {
        for (long long i = threadIdx.x; i < npx; i += blockDim.x) {
            const float v = __ldg(p + i);
            lo = fminf(lo, v);
            hi = fmaxf(hi, v);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __shared__ float slo[32], shi[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { slo[w] = lo; shi[w] = hi; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        lo = l < nw ? slo[l] : FLT_MAX;
        hi = l < nw ? shi[l] : -FLT_MAX;
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (l == 0) {
            const float span = __fsub_rn(hi, lo);
            stats[z] = make_float4(lo, hi, span < 1e-6f ? 1.0f : span, span <= 0.0f ? 1.0f : span);
        }
    }
}

// --------------------------------------------------------------- normalise
// img[zg][y][x] = (v(4zg), v(4zg+1), v(4zg+2), v(4zg+3)) and imgT[zg][x][y], with
// v = (raw - min) * (1 / span_fwd) for raw != 0 and v = 0 for raw == 0: the
// reference skips background pixels (SerialBackend.cpp:104-106). With
// skip_zero = 0 every pixel is normalised, as the reference's CUDA backend does
// (CUDABackend.cu:46-50); imgT may then be null (the ray march reads rows). Both copies
// use the zero-bordered layout of the projector (kFwdGuard pixels left and
// right of every row, kFwdRows rows below the last; a pixel holds the 8 slices
// of a plane pair as two float4, group zg being half zg % 2 of pair zg / 2);
// only the interior is written here, the borders are zeroed when the buffers
// are set up. With box
// set, box[2 zg] = {x min, x max, y min, y max} of the pixels with a non-zero
// value in any slice of the group and box[2 zg + 1].x the largest
// (2x - w + 1)^2 + (2y - h + 1)^2 among them (four times the squared distance
// from the image centre; both emptied by k_slice_stats): the projector walks
// only where its intervals meet that box and that disc, every other pixel
// being an exact zero. With band set, the group's ceil(h/8) row bands (8 rows
// each) get the x range of their non-zero pixels, followed by its ceil(w/8)
// column bands with their y range (emptied by k_slice_stats too).
__global__ void __launch_bounds__(256) k_normalize(const float* __restrict__ vol, int w, int h, int nz,
                                                   const float4* __restrict__ stats,
                                                   float4* __restrict__ img, float4* __restrict__ imgT,
                                                   int skip_zero, int4* __restrict__ box,
                                                   int2* __restrict__ band) {
    const long long pw = w + 2 * kFwdGuard, ph = h + 2 * kFwdGuard;  // row pitches
    const long long rw = h + kFwdRows, rh = w + kFwdRows;             // rows per plane
    __shared__ float4 tile[32][33];
    // the two 4-slice groups of a plane pair run in neighbouring blocks, so
    // both halves of each 32-byte pixel are written at about the same time
    const int zg = 2 * blockIdx.z + (blockIdx.x & 1);
    if (zg >= (nz + 3) / 4) return;  // a pair with one group (uniform per block)
    const int x0 = (blockIdx.x >> 1) * 32, y0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    float lo[4], inv[4];
    bool live[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int z = 4 * zg + j;
        live[j] = z < nz;
        const float4 st = live[j] ? stats[z] : make_float4(0.f, 0.f, 1.f, 1.f);
        lo[j] = st.x;
        inv[j] = __fdiv_rn(1.0f, st.z);
    }
    int bx0 = INT_MAX, bx1 = -1, by0 = INT_MAX, by1 = -1;  // this thread's non-zero pixels
    int r4 = -1;
    int rx[4];  // per row r: this thread's x if its pixel there is non-zero, else -1
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int y = y0 + ty + 8 * r, x = x0 + tx;
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        if (x < w && y < h) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (!live[j]) continue;
                const float raw = __ldg(vol + (static_cast<long long>(4 * zg + j) * h + y) * w + x);
                v[j] = (skip_zero && raw == 0.0f) ? 0.0f : __fmul_rn(__fsub_rn(raw, lo[j]), inv[j]);
            }
        }
        const float4 q = make_float4(v[0], v[1], v[2], v[3]);
        const bool nzp = q.x != 0.0f || q.y != 0.0f || q.z != 0.0f || q.w != 0.0f;
        rx[r] = nzp ? x : -1;
        if (nzp) {
            bx0 = min(bx0, x);
            bx1 = max(bx1, x);
            by0 = min(by0, y);
            by1 = max(by1, y);
            const int dx = 2 * x - w + 1, dy = 2 * y - h + 1;
            r4 = max(r4, dx * dx + dy * dy);
        }
        tile[ty + 8 * r][tx] = q;
        if (x < w && y < h) img[((zg / 2 * rw + y) * pw + x + kFwdGuard) * 2 + (zg & 1)] = q;
    }
    __shared__ int4 wbox[8];  // per warp, then one set of atomics per block
    __shared__ int wr4[8];
    __shared__ int2 srow[4][8];  // [row band of the block][warp]: x range
    __shared__ int2 scol[4][8];  // [column band of the block][warp]: y range
    if (band) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int a = __reduce_min_sync(0xffffffffu, rx[r] >= 0 ? rx[r] : INT_MAX);
            const int b = __reduce_max_sync(0xffffffffu, rx[r]);
            if (tx == 0) srow[r][ty] = make_int2(a, b);
        }
        // this thread's column: y range of its non-zero pixels, reduced over
        // the 8 lanes of its column band
        int c0 = INT_MAX, c1 = -1;
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (rx[r] >= 0) {
                c0 = min(c0, y0 + ty + 8 * r);
                c1 = max(c1, y0 + ty + 8 * r);
            }
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            c0 = min(c0, __shfl_xor_sync(0xffffffffu, c0, o));
            c1 = max(c1, __shfl_xor_sync(0xffffffffu, c1, o));
        }
        if ((tx & 7) == 0) scol[tx >> 3][ty] = make_int2(c0, c1);
    }
    if (box) {
        bx0 = __reduce_min_sync(0xffffffffu, bx0);
        bx1 = __reduce_max_sync(0xffffffffu, bx1);
        by0 = __reduce_min_sync(0xffffffffu, by0);
        by1 = __reduce_max_sync(0xffffffffu, by1);
        r4 = __reduce_max_sync(0xffffffffu, r4);
        if (tx == 0) {
            wbox[ty] = make_int4(bx0, bx1, by0, by1);
            wr4[ty] = r4;
        }
    }
    __syncthreads();
    if (box && threadIdx.x == 0) {
        int4 b = wbox[0];
        int r = wr4[0];
        for (int k = 1; k < 8; ++k) {
            b = make_int4(min(b.x, wbox[k].x), max(b.y, wbox[k].y), min(b.z, wbox[k].z), max(b.w, wbox[k].w));
            r = max(r, wr4[k]);
        }
        if (b.y >= 0) {
            atomicMin(&box[2 * zg].x, b.x);
            atomicMax(&box[2 * zg].y, b.y);
            atomicMin(&box[2 * zg].z, b.z);
            atomicMax(&box[2 * zg].w, b.w);
            atomicMax(&box[2 * zg + 1].x, r);
        }
    }
    if (band && threadIdx.x < 8) {
        // threads 0..3: the block's row bands; 4..7: its column bands
        const int k = threadIdx.x & 3;
        const bool is_row = threadIdx.x < 4;
        int2 b = is_row ? srow[k][0] : scol[k][0];
        for (int t = 1; t < 8; ++t) {
            const int2 c = is_row ? srow[k][t] : scol[k][t];
            b = make_int2(min(b.x, c.x), max(b.y, c.y));
        }
        const int nby = (h + 7) / 8, nbx = (w + 7) / 8;
        const int idx = is_row ? (y0 >> 3) + k : nby + (x0 >> 3) + k;
        if (b.y >= 0 && idx < (is_row ? nby : nby + nbx)) {
            int2* e = band + static_cast<long long>(zg) * (nby + nbx) + idx;
            atomicMin(&e->x, b.x);
            atomicMax(&e->y, b.y);
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int x = x0 + ty + 8 * r, y = y0 + tx;
        if (imgT && x < w && y < h) imgT[((zg / 2 * rh + x) * ph + y + kFwdGuard) * 2 + (zg & 1)] = tile[tx][ty + 8 * r];
    }
}

// ------------------------------------------------------------- ray march
// The reference CUDA backend's forward projector (radonForwardGatherKernel,
// CUDABackend.cu:108-153): the ray of bin b at angle a passes through
// (cx + u cos, cy - u sin), u = b - det_center, with direction (sin, cos);
// samples t = -half + i, i < floor(2 half) + 1 (half = sqrt(w^2 + h^2) / 2),
// each the bilinear interpolation of the normalised image, zero outside. A
// thread owns one (bin, angle) for four slices (one float4 image plane). Only
// samples whose bilinear footprint can touch the image are visited (the
// others add exact zeros in the reference): the parameter range is clipped to
// -1 < x < w, -1 < y < h in double and widened by one sample each side. Pixel
// columns read lie in [-2, w + 1] (inside the zero border); rows above the
// image are skipped explicitly, rows below it are the zero rows of the plane.
__global__ void __launch_bounds__(128) k_raymarch(const float4* __restrict__ img, int w, int h, int nz, int na,
                                                  int nd, float det_center, const double2* __restrict__ cs,
                                                  float* __restrict__ sino) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    const int zg = blockIdx.z;
    if (b >= nd) return;
    const long long pitch = w + 2 * kFwdGuard;
    // group zg is half zg % 2 of the pixels (two float4 each) of plane pair zg / 2
    const float4* plane = img + static_cast<long long>(zg / 2) * (h + kFwdRows) * pitch * 2 + 2 * kFwdGuard + (zg & 1);
    const double2 tc = cs[a];
    const float c = static_cast<float>(tc.x), s = static_cast<float>(tc.y);
    const float cx = 0.5f * static_cast<float>(w - 1), cy = 0.5f * static_cast<float>(h - 1);
    const float u = static_cast<float>(b) - det_center;
    const float bx = cx + u * c, by = cy - u * s;
    const float half = 0.5f * sqrtf(static_cast<float>(w * w + h * h));
    const int ns = static_cast<int>(2.0f * half) + 1;
    // parameter range with -1 < x(t) < w and -1 < y(t) < h
    double tlo = -1e30, thi = 1e30;
    const double sd = s, cd = c;
    if (fabs(sd) > 1e-12) {
        const double t0 = (-1.0 - bx) / sd, t1 = (w - static_cast<double>(bx)) / sd;
        tlo = fmax(tlo, fmin(t0, t1));
        thi = fmin(thi, fmax(t0, t1));
    } else if (!(bx > -1.0f && bx < static_cast<float>(w))) {
        thi = -2e30;
    }
    if (fabs(cd) > 1e-12) {
        const double t0 = (-1.0 - by) / cd, t1 = (h - static_cast<double>(by)) / cd;
        tlo = fmax(tlo, fmin(t0, t1));
        thi = fmin(thi, fmax(t0, t1));
    } else if (!(by > -1.0f && by < static_cast<float>(h))) {
        thi = -2e30;
    }
    float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
    if (thi >= tlo) {
        const int i0 = max(0, static_cast<int>(floor(tlo + half)) - 1);
        const int i1 = min(ns - 1, static_cast<int>(ceil(thi + half)) + 1);
        for (int i = i0; i <= i1; ++i) {
            const float t = static_cast<float>(i) - half;
            const float x = bx + t * s, y = by + t * c;
            const float xf = floorf(x), yf = floorf(y);
            const int x0 = static_cast<int>(xf), y0 = static_cast<int>(yf);
            const float fx = x - xf, fy = y - yf;
            const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
            const float4* r0 = plane + 2 * (static_cast<long long>(y0) * pitch + x0);
            const float4 v00 = y0 >= 0 ? r0[0] : zero, v10 = y0 >= 0 ? r0[2] : zero;
            const float4 v01 = y0 + 1 >= 0 ? r0[2 * pitch] : zero, v11 = y0 + 1 >= 0 ? r0[2 * pitch + 2] : zero;
            const float w00 = (1.0f - fx) * (1.0f - fy), w10 = fx * (1.0f - fy);
            const float w01 = (1.0f - fx) * fy, w11 = fx * fy;
            sum.x += w00 * v00.x + w10 * v10.x + w01 * v01.x + w11 * v11.x;
            sum.y += w00 * v00.y + w10 * v10.y + w01 * v01.y + w11 * v11.y;
            sum.z += w00 * v00.z + w10 * v10.z + w01 * v01.z + w11 * v11.z;
            sum.w += w00 * v00.w + w10 * v10.w + w01 * v01.w + w11 * v11.w;
        }
    }
    const float v[4] = {sum.x, sum.y, sum.z, sum.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int z = 4 * zg + j;
        if (z < nz) sino[(static_cast<long long>(z) * na + a) * nd + b] = v[j];
    }
}

}  // namespace

cudaError_t launch_raymarch(const float4* d_img, int w, int h, int nz, int na, int nd, float det_center,
                            const double2* d_cs, float* d_sino, cudaStream_t st) {
    const dim3 grid((nd + 127) / 128, na, (nz + 3) / 4);
    k_raymarch<<<grid, 128, 0, st>>>(d_img, w, h, nz, na, nd, det_center, d_cs, d_sino);
    return cudaGetLastError();
}

cudaError_t launch_trig(const float* d_angles_deg, int na, double2* d_cs, cudaStream_t st) {
    k_trig<<<(na + 127) / 128, 128, 0, st>>>(d_angles_deg, na, d_cs);
    return cudaGetLastError();
}

cudaError_t launch_slice_stats(const float* d_vol, long long npx, int nz, float4* d_stats,
                               cudaStream_t st, int4* d_box, int2* d_band, int nband) {
    k_slice_stats<<<nz, 1024, 0, st>>>(d_vol, npx, d_stats, d_box, d_band, nband);
    return cudaGetLastError();
}

cudaError_t launch_normalize(const float* d_vol, int w, int h, int nz, const float4* d_stats,
                             float4* d_img, float4* d_imgT, cudaStream_t st, int skip_zero,
                             int4* d_box, int2* d_band) {
    const dim3 grid(2 * ((w + 31) / 32), (h + 31) / 32, (nz + 7) / 8);
    k_normalize<<<grid, 256, 0, st>>>(d_vol, w, h, nz, d_stats, d_img, d_imgT, skip_zero, d_box, d_band);
    return cudaGetLastError();
}

}  // namespace ctb
