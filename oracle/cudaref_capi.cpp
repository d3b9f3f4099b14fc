// cudaref_capi.cpp — TEST INFRASTRUCTURE, not product code.
//
// A thin extern "C" layer over the reference's own CUDA backend
// (CUDABackend.cu), compiled with it and the reference CPU sources it needs by
// oracle/Makefile into oracle/_ref/libctref_cuda.so. It pins the oracle's
// restatement of the CUDA backend's conventions (ray-march forward projector,
// (N-1)/2 centres, Nyquist-keeping filter) against the reference itself, run
// once on a GPU to write tests/golden/cuda_conv.npz. It reimplements nothing:
// every function forwards to CUDABackend.

#include "CUDABackend.h"

#include <cstring>
#include <vector>

using namespace ct;

extern "C" {

// CUDABackend::computeSinogram (CUDABackend.cu:524-590).
int cref_compute_sinogram(const float* slice, int w, int h, int na, int nd, float* sino, float* minmax) {
    CUDABackend be;
    if (!be.isAvailable()) return 2;
    Buffer2D s(static_cast<size_t>(w), static_cast<size_t>(h));
    std::memcpy(s.data.data(), slice, sizeof(float) * s.data.size());
    const Sinogram out = be.computeSinogram(s, static_cast<size_t>(na), static_cast<size_t>(nd), true);
    if (out.data.data.size() != static_cast<size_t>(na) * nd) return 1;
    std::memcpy(sino, out.data.data.data(), sizeof(float) * out.data.data.size());
    if (minmax) {
        minmax[0] = out.original_min_hu;
        minmax[1] = out.original_max_hu;
    }
    return 0;
}

// CUDABackend::reconstructSlice (CUDABackend.cu:592-690); min/max as the
// Sinogram's original_min_hu / original_max_hu (denormalised when max > min).
int cref_reconstruct_slice(const float* sino, int na, int nd, const float* angles_deg, int n_out, int filter,
                           float min_hu, float max_hu, float* out) {
    CUDABackend be;
    if (!be.isAvailable()) return 2;
    Sinogram s;
    s.data.assign(static_cast<size_t>(nd), static_cast<size_t>(na), 0.0f);
    std::memcpy(s.data.data.data(), sino, sizeof(float) * static_cast<size_t>(na) * nd);
    s.angles_deg.assign(angles_deg, angles_deg + na);
    s.original_min_hu = min_hu;
    s.original_max_hu = max_hu;
    ReconstructionParams p;
    p.filter = static_cast<ReconstructionParams::FilterType>(filter);
    p.num_angles = static_cast<size_t>(na);
    const Buffer2D r = be.reconstructSlice(s, static_cast<size_t>(n_out), p);
    if (r.data.size() != static_cast<size_t>(n_out) * n_out) return 1;
    std::memcpy(out, r.data.data(), sizeof(float) * r.data.size());
    return 0;
}

// CUDABackend::reconstructVolume (CUDABackend.cu:692-...): vol and out n x n x depth.
int cref_reconstruct_volume(const float* vol, int n, int depth, int na, int filter, float* out) {
    CUDABackend be;
    if (!be.isAvailable()) return 2;
    Volume in;
    in.assign(static_cast<size_t>(n), static_cast<size_t>(n), static_cast<size_t>(depth), 0.0f);
    std::memcpy(in.data.data(), vol, sizeof(float) * in.data.size());
    Volume res;
    ReconstructionParams p;
    p.filter = static_cast<ReconstructionParams::FilterType>(filter);
    p.num_angles = static_cast<size_t>(na);
    be.reconstructVolume(in, res, p, nullptr);
    if (res.data.size() != in.data.size()) return 1;
    std::memcpy(out, res.data.data(), sizeof(float) * res.data.size());
    return 0;
}

}  // extern "C"
