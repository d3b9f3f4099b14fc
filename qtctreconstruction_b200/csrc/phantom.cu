// phantom.cu — ellipsoid phantoms (the Generator3D data source of the path,
// Generator3D.h:12-47) and the threshold point-cloud compaction
// (IReconstructionBackend::extractPointCloud, SerialBackend.cpp:325-346).
//
// Two generator modes:
//  * k_phantom_sum — the benchmark phantom: rotated ellipsoids with summed
//    densities, zero outside the unit sphere. Voxel coordinates are
//    (2i - (n-1)) / n per axis. Every product and sum is rounded separately
//    (explicit _rn intrinsics, no fused multiply-add) in a fixed order, so
//    the result is bit-identical to the CPU restatement.
//  * k_generator3d — Generator3DCPU's model (Generator3DCPU.cpp:67-117):
//    axis-aligned ellipsoids in millimetre coordinates from linspace, max
//    compositing over -1000 HU, the same float expressions and divisions.
// Both cull ellipsoids per CTA tile with conservative index-space boxes
// computed on the host; culling only skips ellipsoids that cannot contain a
// voxel of the tile, so sums keep their order and maxima their value.
#include <cfloat>

#include "ctb_internal.h"

namespace ctb {
namespace {

constexpr int TX = 32, TY = 8, TZ = 4;  // CTA tile: 32 x 8 x 4 voxels, 256 threads
constexpr int TZS = 8;                  // k_phantom_sum: 32 x 8 x 8 voxels, 8 slices per thread
constexpr int MAXC = 1024;              // candidate list capacity per CTA

// Ordered compaction of the ellipsoids whose box meets the tile.
// boxes: 6 ints per ellipsoid {x0, x1, y0, y1, z0, z1} (inclusive).
__device__ int cull(const int* __restrict__ boxes, int k, int x0, int y0, int z0,
                    short* cand, int* warp_tot, int tz = TZ) {
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    int total = 0;
    for (int base = 0; base < k; base += blockDim.x) {
        const int e = base + t;
        bool hit = false;
        if (e < k) {
            const int* b = boxes + 6 * e;
            hit = !(b[1] < x0 || b[0] > x0 + TX - 1 || b[3] < y0 || b[2] > y0 + TY - 1 ||
                    b[5] < z0 || b[4] > z0 + tz - 1);
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) warp_tot[wid] = __popc(m);
        __syncthreads();
        int off = total;
        for (int w = 0; w < wid; ++w) off += warp_tot[w];
        if (hit) {
            const int pos = off + __popc(m & ((1u << lane) - 1u));
            if (pos < MAXC) cand[pos] = static_cast<short>(e);
        }
        int sum = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += warp_tot[w];
        total += sum;
        __syncthreads();
    }
    return total;
}

__device__ __forceinline__ float grid_coord(int i, int n) {
    return __fdiv_rn(__fsub_rn(__fmul_rn(2.0f, static_cast<float>(i)), static_cast<float>(n - 1)),
                     static_cast<float>(n));
}

// One ellipsoid staged for k_phantom_sum: the coefficients of the terms in x
// and y (the same for a thread's 8 slices) as scalars, those that meet the
// slice coordinate as duplicated pairs for the packed FP32x2 instructions.
struct PhEll {
    float cx, cy, r00, r01, r10, r11, r20, r21;         // p0 p1 p3 p4 p6 p7 p9 p10
    float2 cz, r02, r12, r22, i0, i1, i2, dens;          // p2 p5 p8 p11 p12 p13 p14 p15, each twice
};

// a - b as one packed instruction: fma(b, -1, a) rounds a - b exactly once
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}

// Every thread holds one (x, y) column of TZS slices; the slice terms run two
// slices per packed FP32x2 instruction. Each lane of a packed add or multiply
// is the IEEE round-to-nearest result of the scalar operation, in the same
// order as the scalar code of the oracle, so the phantom stays bit-identical.
__global__ void __launch_bounds__(256) k_phantom_sum(const float* __restrict__ params,
                                                     const int* __restrict__ boxes, int k, int nx,
                                                     int ny, int nz, float* __restrict__ vol) {
    __shared__ short cand[MAXC];
    __shared__ int warp_tot[8];
    __shared__ PhEll sp[64];
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZS;
    // A tile whose voxel nearest the centre lies outside the unit sphere holds
    // only zeros: the rounded r^2 below grows with every |coordinate|, so no
    // voxel of the tile passes r2 <= 1 (the test is the voxels' own expression
    // on coordinates no larger than theirs). Such tiles skip the ellipsoids.
    const bool outside = [&] {
        auto nearest = [](int lo, int len, int n) {
            const int hi = min(lo + len, n) - 1;
            if (2 * hi < n - 1) return fabsf(grid_coord(hi, n));
            if (2 * lo > n - 1) return fabsf(grid_coord(lo, n));
            return 0.0f;  // the tile straddles the centre plane
        };
        const float mx = nearest(x0, TX, nx), my = nearest(y0, TY, ny), mz = nearest(z0, TZS, nz);
        return __fadd_rn(__fadd_rn(__fmul_rn(mx, mx), __fmul_rn(my, my)), __fmul_rn(mz, mz)) > 1.0f;
    }();
    const int nc = outside ? 0 : cull(boxes, k, x0, y0, z0, cand, warp_tot, TZS);
    const bool overflow = nc > MAXC;  // fall back to every ellipsoid
    const int ncand = overflow ? k : nc;
    const int x = x0 + (threadIdx.x & 31), y = y0 + (threadIdx.x >> 5);
    const bool live_xy = x < nx && y < ny;
    const float X = grid_coord(x, nx), Y = grid_coord(y, ny);
    constexpr int NPAIR = TZS / 2;
    float acc[TZS];
    float2 Z[NPAIR];
    bool in[TZS];
#pragma unroll
    for (int j = 0; j < TZS; ++j) {
        acc[j] = 0.0f;
        const float zj = grid_coord(z0 + j, nz);
        if (j & 1) Z[j / 2].y = zj;
        else Z[j / 2].x = zj;
        const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(X, X), __fmul_rn(Y, Y)), __fmul_rn(zj, zj));
        in[j] = r2 <= 1.0f;
    }
    for (int base = 0; base < ncand; base += 64) {
        const int cnt = min(64, ncand - base);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
            const int e = overflow ? base + i : cand[base + i];
            const float* p = params + 16 * e;
            PhEll q;
            q.cx = p[0];
            q.cy = p[1];
            q.r00 = p[3];
            q.r01 = p[4];
            q.r10 = p[6];
            q.r11 = p[7];
            q.r20 = p[9];
            q.r21 = p[10];
            q.cz = make_float2(p[2], p[2]);
            q.r02 = make_float2(p[5], p[5]);
            q.r12 = make_float2(p[8], p[8]);
            q.r22 = make_float2(p[11], p[11]);
            q.i0 = make_float2(p[12], p[12]);
            q.i1 = make_float2(p[13], p[13]);
            q.i2 = make_float2(p[14], p[14]);
            q.dens = make_float2(p[15], p[15]);
            sp[i] = q;
        }
        __syncthreads();
        for (int c = 0; c < cnt; ++c) {
            const PhEll& q = sp[c];
            const float dx = __fsub_rn(X, q.cx), dy = __fsub_rn(Y, q.cy);
            // the x and y terms of the three body coordinates, shared by the slices
            const float u0 = __fadd_rn(__fmul_rn(q.r00, dx), __fmul_rn(q.r01, dy));
            const float u1 = __fadd_rn(__fmul_rn(q.r10, dx), __fmul_rn(q.r11, dy));
            const float u2 = __fadd_rn(__fmul_rn(q.r20, dx), __fmul_rn(q.r21, dy));
            const float2 U0 = make_float2(u0, u0), U1 = make_float2(u1, u1), U2 = make_float2(u2, u2);
#pragma unroll
            for (int h = 0; h < NPAIR; ++h) {
                const float2 dz = sub2(Z[h], q.cz);
                const float2 b0 = __fadd2_rn(U0, __fmul2_rn(q.r02, dz));
                const float2 b1 = __fadd2_rn(U1, __fmul2_rn(q.r12, dz));
                const float2 b2 = __fadd2_rn(U2, __fmul2_rn(q.r22, dz));
                const float2 qq = __fadd2_rn(__fadd2_rn(__fmul2_rn(__fmul2_rn(b0, b0), q.i0),
                                                        __fmul2_rn(__fmul2_rn(b1, b1), q.i1)),
                                             __fmul2_rn(__fmul2_rn(b2, b2), q.i2));
                if (in[2 * h] && qq.x <= 1.0f) acc[2 * h] = __fadd_rn(acc[2 * h], q.dens.x);
                if (in[2 * h + 1] && qq.y <= 1.0f) acc[2 * h + 1] = __fadd_rn(acc[2 * h + 1], q.dens.y);
            }
        }
    }
    if (!live_xy) return;
#pragma unroll
    for (int j = 0; j < TZS; ++j) {
        const int z = z0 + j;
        if (z < nz) vol[(static_cast<long long>(z) * ny + y) * nx + x] = acc[j];
    }
}

// linspace(-r, r, n)[i] as Utils.cpp:9-22 computes it: start + step * i.
__device__ __forceinline__ float lin(float r, int n, int i) {
    if (n == 1) return -r;
    const float step = __fdiv_rn(__fsub_rn(r, -r), static_cast<float>(n - 1));
    return __fadd_rn(-r, __fmul_rn(step, static_cast<float>(i)));
}

// ell: 7 floats per ellipsoid {cx, cy, cz, ax, ay, az, hu} in millimetres.
__global__ void __launch_bounds__(256) k_generator3d(const float* __restrict__ ell,
                                                     const int* __restrict__ boxes, int k, int nx,
                                                     int ny, int nz, float radius,
                                                     float* __restrict__ vol) {
    __shared__ short cand[MAXC];
    __shared__ int warp_tot[8];
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
    const int nc = cull(boxes, k, x0, y0, z0, cand, warp_tot);
    const bool overflow = nc > MAXC;
    const int ncand = overflow ? k : nc;
    const int x = x0 + (threadIdx.x & 31), y = y0 + (threadIdx.x >> 5);
    if (x >= nx || y >= ny) return;
    const float xs = lin(radius, nx, x), ys = lin(radius, ny, y);
    for (int j = 0; j < TZ; ++j) {
        const int z = z0 + j;
        if (z >= nz) break;
        const float zs = lin(radius, nz, z);
        float v = -1000.0f;
        for (int c = 0; c < ncand; ++c) {
            const float* p = ell + 7 * (overflow ? c : cand[c]);
            const float dx = __fsub_rn(xs, p[0]), dy = __fsub_rn(ys, p[1]), dz = __fsub_rn(zs, p[2]);
            const float t0 = __fdiv_rn(__fmul_rn(dx, dx), __fmul_rn(p[3], p[3]));
            const float t1 = __fdiv_rn(__fmul_rn(dy, dy), __fmul_rn(p[4], p[4]));
            const float t2 = __fdiv_rn(__fmul_rn(dz, dz), __fmul_rn(p[5], p[5]));
            if (__fadd_rn(__fadd_rn(t0, t1), t2) <= 1.0f) v = fmaxf(v, p[6]);
        }
        vol[(static_cast<long long>(z) * ny + y) * nx + x] = v;
    }
}

// ------------------------------------------------------------ point cloud
constexpr int PC_THREADS = 256;
constexpr int PC_PER_BLOCK = 4096;

__global__ void __launch_bounds__(PC_THREADS) k_point_count(const float* __restrict__ vol,
                                                            long long total, float thr,
                                                            unsigned* __restrict__ counts) {
    const long long base = static_cast<long long>(blockIdx.x) * PC_PER_BLOCK;
    unsigned c = 0;
    for (int i = threadIdx.x; i < PC_PER_BLOCK; i += PC_THREADS) {
        const long long g = base + i;
        if (g < total && vol[g] > thr) ++c;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ unsigned ws[PC_THREADS / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned s = 0;
        for (int w = 0; w < PC_THREADS / 32; ++w) s += ws[w];
        counts[blockIdx.x] = s;
    }
}

// Writes the points of each block in index order at the block's offset.
__global__ void __launch_bounds__(PC_THREADS) k_point_write(
    const float* __restrict__ vol, int nx, int ny, long long total, float thr,
    const unsigned long long* __restrict__ offsets, float4* __restrict__ pts, long long cap) {
    const long long base = static_cast<long long>(blockIdx.x) * PC_PER_BLOCK;
    __shared__ unsigned ws[PC_THREADS / 32];
    unsigned long long run = offsets[blockIdx.x];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i0 = 0; i0 < PC_PER_BLOCK; i0 += PC_THREADS) {
        const long long g = base + i0 + threadIdx.x;
        const float v = g < total ? vol[g] : 0.0f;
        const bool hit = g < total && v > thr;
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) ws[wid] = __popc(m);
        __syncthreads();
        unsigned off = 0, sum = 0;
        for (int w = 0; w < PC_THREADS / 32; ++w) {
            if (w < wid) off += ws[w];
            sum += ws[w];
        }
        if (hit) {
            const unsigned long long pos = run + off + __popc(m & ((1u << lane) - 1u));
            if (static_cast<long long>(pos) < cap) {
                const long long x = g % nx, yz = g / nx;
                const long long y = yz % ny, z = yz / ny;
                pts[pos] = make_float4(static_cast<float>(x), static_cast<float>(y),
                                       static_cast<float>(z), v);
            }
        }
        run += sum;
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_phantom_sum_boxes(const float* d_params, const int* d_boxes, int k, int nx,
                                     int ny, int nz, float* d_vol, cudaStream_t st) {
    const dim3 grid((nx + TX - 1) / TX, (ny + TY - 1) / TY, (nz + TZS - 1) / TZS);
    k_phantom_sum<<<grid, 256, 0, st>>>(d_params, d_boxes, k, nx, ny, nz, d_vol);
    return cudaGetLastError();
}

cudaError_t launch_generator3d_boxes(const float* d_ell, const int* d_boxes, int k, int nx,
                                     int ny, int nz, float radius_mm, float* d_vol,
                                     cudaStream_t st) {
    const dim3 grid((nx + TX - 1) / TX, (ny + TY - 1) / TY, (nz + TZ - 1) / TZ);
    k_generator3d<<<grid, 256, 0, st>>>(d_ell, d_boxes, k, nx, ny, nz, radius_mm, d_vol);
    return cudaGetLastError();
}

int point_blocks(long long total) {
    return static_cast<int>((total + PC_PER_BLOCK - 1) / PC_PER_BLOCK);
}

cudaError_t launch_point_count(const float* d_vol, long long total, float thr,
                               unsigned* d_block_counts, int blocks, cudaStream_t st) {
    k_point_count<<<blocks, PC_THREADS, 0, st>>>(d_vol, total, thr, d_block_counts);
    return cudaGetLastError();
}

cudaError_t launch_point_write(const float* d_vol, int nx, int ny, long long total, float thr,
                               const unsigned long long* d_block_offsets, int blocks,
                               float4* d_points, long long cap, cudaStream_t st) {
    k_point_write<<<blocks, PC_THREADS, 0, st>>>(d_vol, nx, ny, total, thr, d_block_offsets,
                                                 d_points, cap);
    return cudaGetLastError();
}

}  // namespace ctb
