// probe.cu — shared-memory load bandwidth probe (the roofline denominator of
// the backprojector, whose inner loop is bound by 16-byte shared loads).
//
// Every thread streams float4 loads from a shared buffer at a lane-contiguous,
// conflict-free address pattern and folds them into an accumulator that is
// stored at the end (so the loads cannot be removed). Bytes moved = blocks x
// threads x iterations x 16.
#include "ctb_internal.h"

namespace ctb {
namespace {

constexpr int PROBE_THREADS = 512;
constexpr int PROBE_ITERS = 4096;

__global__ void __launch_bounds__(PROBE_THREADS) k_smem_probe(float* out) {
    __shared__ float4 buf[2048];
    for (int i = threadIdx.x; i < 2048; i += blockDim.x)
        buf[i] = make_float4(i * 1.0f, i * 0.5f, i * 0.25f, i * 0.125f);
    __syncthreads();
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    int idx = threadIdx.x & 2047;
#pragma unroll 16
    for (int it = 0; it < PROBE_ITERS; ++it) {
        const float4 v = buf[idx];
        acc.x += v.x;
        acc.y += v.y;
        acc.z += v.z;
        acc.w += v.w;
        idx = (idx + 32) & 2047;
    }
    if (acc.x + acc.y + acc.z + acc.w == 1234.5f) out[blockIdx.x] = acc.x;
}

}  // namespace

cudaError_t smem_probe(int sms, float* d_out, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1,
                       double* bytes) {
    const int blocks = sms * 4;
    k_smem_probe<<<blocks, PROBE_THREADS, 0, st>>>(d_out);  // warm-up
    cudaEventRecord(e0, st);
    k_smem_probe<<<blocks, PROBE_THREADS, 0, st>>>(d_out);
    cudaEventRecord(e1, st);
    *bytes = static_cast<double>(blocks) * PROBE_THREADS * PROBE_ITERS * 16.0;
    return cudaGetLastError();
}

}  // namespace ctb
