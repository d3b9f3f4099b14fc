// noalloc.cu — ctb_fbp_noalloc: filtered backprojection of up to four slices
// that allocates no device memory.
//
// Some callers cannot allocate device memory at the point where they need a
// reconstruction: code running under a caller-owned memory pool that forbids
// outside allocations, real-time loops that must not stall on the allocator,
// or hosts whose allocator is not cudaMalloc at all. For them this entry point
// takes device buffers for the input and the output only; every intermediate
// (angle tables, filter spectrum, twiddles, filtered rows, the device error
// word) lives in one file-scope static device array of kScratchBytes, which
// each GPU that loads the library holds until the process exits.
//
// The host never uses the array's name as an address (in host code it is only
// a stand-in symbol): the device address is looked up once per device with
// cudaGetSymbolAddress, on the first call made on that device, and cached.
// Make that first call before any stream capture. Every call shares the
// array and leaves its contents behind; what must start at zero (the error
// word) is cleared on every call, and two calls that overlap on the GPU (two
// host threads, or two streams) race on the array.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "ctb_internal.h"

namespace {

// Fixed layout of the scratch array (all offsets 256-byte aligned).
constexpr int kMaxAngles = 2048;
constexpr int kMaxConv = 8192;                       // convolution length Lc
constexpr size_t kScratchBytes = size_t(16) << 20;  // 16 MiB
constexpr size_t kOffErr = 0;
constexpr size_t kOffAngles = 256;
constexpr size_t kOffTrig = kOffAngles + sizeof(float) * kMaxAngles;           // double2 + float2
constexpr size_t kOffHc = kOffTrig + (sizeof(double2) + sizeof(float2)) * kMaxAngles;
// The filter spectrum (filter_table): Lc float2, plus Lc packed float4 when
// Lc <= 2048, so at most max(8192, 3 x 2048) = 8192 float2.
constexpr size_t kHcEntries = kMaxConv;
static_assert(3 * 2048 <= kHcEntries, "spectrum region too small");
constexpr size_t kOffTw = kOffHc + sizeof(float2) * kHcEntries;
// FFT twiddle tables (fft_twiddle_table): the longest is that of Lc = 8192,
// 15 (8192/8 - 1) + 4096 = 19441 float2 (Lc = 2048 with its packed copy takes
// 3 x 5617 + 1). Rounded up to 256 bytes.
constexpr size_t kTwEntries = 15 * (kMaxConv / 8 - 1) + kMaxConv / 2;
static_assert(3 * (15 * (2048 / 8 - 1) + 7 * (2048 / 8)) + 1 <= kTwEntries, "twiddle region too small");
constexpr size_t kOffFilt = kOffTw + (sizeof(float2) * kTwEntries + 255) / 256 * 256;
constexpr size_t kFiltCapacity = (kScratchBytes - kOffFilt) / sizeof(float4);  // float4 bins
static_assert(kOffTrig % 256 == 0 && kOffHc % 256 == 0 && kOffTw % 256 == 0 && kOffFilt % 256 == 0,
              "scratch layout must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch per device, looked up once.
std::mutex g_mu;
std::vector<unsigned char*> g_addr;

ctb_status scratch_address(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CTB_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    if (static_cast<int>(g_addr.size()) <= dev) g_addr.resize(dev + 1, nullptr);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return CTB_ERR_CUDA;
        }
        g_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[dev];
    return CTB_OK;
}

}  // namespace

extern "C" ctb_status ctb_fbp_noalloc(const float* d_sino, int depth, int num_angles, int bins,
                                      const float* angles_deg, int output_size, int filter,
                                      float* d_out, void* stream) {
    using namespace ctb;
    if (!d_sino || !d_out || depth <= 0 || num_angles <= 0 || bins <= 0 || output_size <= 0 ||
        filter < CTB_FILTER_RAMP || filter > CTB_FILTER_BARTLETT)
        return CTB_ERR_INVALID;
    const PadGeom g = pad_geometry(bins);
    const FiltLayout fl = filt_layout(g.sq, output_size);
    // sizes beyond the static scratch are refused, never truncated
    if (depth > 4 || num_angles > kMaxAngles || g.Lc > kMaxConv ||
        static_cast<size_t>(num_angles) * fl.pitch > kFiltCapacity)
        return CTB_ERR_UNSUPPORTED;
    unsigned char* base = nullptr;
    const ctb_status s = scratch_address(&base);
    if (s != CTB_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // host-side tables (double precision), then copies into the scratch
    std::vector<float> deg(num_angles);
    if (angles_deg) {
        std::memcpy(deg.data(), angles_deg, sizeof(float) * num_angles);
    } else {
        const float step = 180.0f / static_cast<float>(num_angles);
        for (int a = 0; a < num_angles; ++a) deg[a] = step * static_cast<float>(a);
    }
    std::vector<float2> csf(num_angles);
    for (int a = 0; a < num_angles; ++a) {
        const float th = deg[a] * 3.14159265358979323846f / 180.0f;
        csf[a] = make_float2(std::cos(th), std::sin(th));
    }
    const std::vector<float2> Hc = filter_table(g, filter);
    const std::vector<float2> tw = fft_twiddle_table(g.Lc);
    if (Hc.size() > kHcEntries || tw.size() > kTwEntries) return CTB_ERR_UNSUPPORTED;
    unsigned* d_err = reinterpret_cast<unsigned*>(base + kOffErr);
    float* d_deg = reinterpret_cast<float*>(base + kOffAngles);
    double2* d_cs = reinterpret_cast<double2*>(base + kOffTrig);
    float2* d_csf = reinterpret_cast<float2*>(d_cs + num_angles);
    float2* d_Hc = reinterpret_cast<float2*>(base + kOffHc);
    float2* d_tw = reinterpret_cast<float2*>(base + kOffTw);
    float4* d_filt = reinterpret_cast<float4*>(base + kOffFilt);

    cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_deg, deg.data(), sizeof(float) * num_angles, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_csf, csf.data(), sizeof(float2) * num_angles, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_Hc, Hc.data(), sizeof(float2) * Hc.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_trig(d_deg, num_angles, d_cs, st);
    const float scale = 3.14159265358979323846f / (2.0f * static_cast<float>(num_angles));
    if (e == cudaSuccess)
        e = launch_filter(d_sino, depth, num_angles, g, fl, d_Hc, d_tw, nullptr, CTB_DENORM_NONE, scale,
                          d_filt, st);
    Trig trig;
    trig.cs = d_cs;
    trig.csf = d_csf;
    if (e == cudaSuccess)
        e = launch_backproject(d_filt, depth, num_angles, fl, output_size, trig, nullptr,
                               CTB_DENORM_NONE, d_out, d_err, st);
    // the host vectors above must outlive the queued copies, and a bounded
    // device wait that gave up is reported through the error word
    unsigned h_err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof h_err, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaStreamSynchronize(st);  // nothing queued may outlive the host tables above
        cudaGetLastError();
        return CTB_ERR_CUDA;
    }
    return h_err ? CTB_ERR_TIMEOUT : CTB_OK;
}
