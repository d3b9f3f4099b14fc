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
constexpr int MAXC = 1024;              // candidate list capacity per CTA

// Ordered compaction of the ellipsoids whose box meets the tile.
// boxes: 6 ints per ellipsoid {x0, x1, y0, y1, z0, z1} (inclusive).
__device__ int cull(const int* __restrict__ boxes, int k, int x0, int y0, int z0,
                    short* cand, int* warp_tot) {
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    int total = 0;
    for (int base = 0; base < k; base += blockDim.x) {
        const int e = base + t;
        bool hit = false;
        if (e < k) {
            const int* b = boxes + 6 * e;
            hit = !(b[1] < x0 || b[0] > x0 + TX - 1 || b[3] < y0 || b[2] > y0 + TY - 1 ||
                    b[5] < z0 || b[4] > z0 + TZ - 1);
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

__global__ void __launch_bounds__(256) k_phantom_sum(const float* __restrict__ params,
                                                     const int* __restrict__ boxes, int k, int nx,
                                                     int ny, int nz, float* __restrict__ vol) {
    __shared__ short cand[MAXC];
    __shared__ int warp_tot[8];
    __shared__ float sp[64][16];
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
    const int nc = cull(boxes, k, x0, y0, z0, cand, warp_tot);
    const bool overflow = nc > MAXC;  // fall back to every ellipsoid
    const int ncand = overflow ? k : nc;
    const int x = x0 + (threadIdx.x & 31), y = y0 + (threadIdx.x >> 5);
    const bool live_xy = x < nx && y < ny;
    const float X = grid_coord(x, nx), Y = grid_coord(y, ny);
    float acc[TZ];
    float Z[TZ];
    bool in[TZ];
#pragma unroll
    for (int j = 0; j < TZ; ++j) {
        acc[j] = 0.0f;
        Z[j] = grid_coord(z0 + j, nz);
        const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(X, X), __fmul_rn(Y, Y)), __fmul_rn(Z[j], Z[j]));
        in[j] = r2 <= 1.0f;
    }
    for (int base = 0; base < ncand; base += 64) {
        const int cnt = min(64, ncand - base);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt * 16; i += blockDim.x) {
            const int e = overflow ? base + i / 16 : cand[base + i / 16];
            sp[i / 16][i % 16] = params[16 * e + (i % 16)];
        }
        __syncthreads();
        for (int c = 0; c < cnt; ++c) {
            const float* p = sp[c];
            const float dx = __fsub_rn(X, p[0]), dy = __fsub_rn(Y, p[1]);
#pragma unroll
            for (int j = 0; j < TZ; ++j) {
                const float dz = __fsub_rn(Z[j], p[2]);
                const float b0 = __fadd_rn(__fadd_rn(__fmul_rn(p[3], dx), __fmul_rn(p[4], dy)), __fmul_rn(p[5], dz));
                const float b1 = __fadd_rn(__fadd_rn(__fmul_rn(p[6], dx), __fmul_rn(p[7], dy)), __fmul_rn(p[8], dz));
                const float b2 = __fadd_rn(__fadd_rn(__fmul_rn(p[9], dx), __fmul_rn(p[10], dy)), __fmul_rn(p[11], dz));
                const float q = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(b0, b0), p[12]),
                                                    __fmul_rn(__fmul_rn(b1, b1), p[13])),
                                          __fmul_rn(__fmul_rn(b2, b2), p[14]));
                if (in[j] && q <= 1.0f) acc[j] = __fadd_rn(acc[j], p[15]);
            }
        }
    }
    if (!live_xy) return;
#pragma unroll
    for (int j = 0; j < TZ; ++j) {
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
    const dim3 grid((nx + TX - 1) / TX, (ny + TY - 1) / TY, (nz + TZ - 1) / TZ);
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
