// ref_capi.cpp — TEST INFRASTRUCTURE, not product code.
//
// A thin extern "C" layer over the reference's own CPU backends, compiled
// together with the unmodified reference sources by oracle/Makefile into
// oracle/_ref/libctref.so. It lets the Python tests and the CPU-baseline leg
// of bench.py call SerialBackend / OpenMPBackend / FilterDesign /
// Generator3DCPU through ctypes. It reimplements nothing: every function
// forwards to the reference class named beside it.

#include "IReconstructionBackend.h"
#include "SerialBackend.h"
#include "OpenMPBackend.h"
#include "FilterDesign.h"
#include "Generator3D.h"
#include "Generator3DCPU.h"

#include <omp.h>

#include <cstring>
#include <memory>
#include <vector>

using namespace ct;

namespace {

std::unique_ptr<IReconstructionBackend> make_backend(int which) {
    if (which == 0) return std::make_unique<SerialBackend>();
    return std::make_unique<OpenMPBackend>();
}

ReconstructionParams params_for(int filter, int na) {
    ReconstructionParams p;
    p.filter = static_cast<ReconstructionParams::FilterType>(filter);
    p.num_angles = static_cast<size_t>(na);
    return p;
}

}  // namespace

extern "C" {

void ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int ref_max_threads() { return omp_get_max_threads(); }

// which: 0 = SerialBackend, 1 = OpenMPBackend.
// IReconstructionBackend::computeSinogram (IReconstructionBackend.h:21).
int ref_compute_sinogram(int which, const float* slice, int w, int h, int na, int nd,
                         float* sino, float* angles_deg, float* minmax) {
    auto be = make_backend(which);
    Buffer2D s(static_cast<size_t>(w), static_cast<size_t>(h));
    std::memcpy(s.data.data(), slice, sizeof(float) * s.data.size());
    const Sinogram out = be->computeSinogram(s, static_cast<size_t>(na), static_cast<size_t>(nd), true);
    if (out.data.data.size() != static_cast<size_t>(na) * nd) return 1;
    std::memcpy(sino, out.data.data.data(), sizeof(float) * out.data.data.size());
    if (angles_deg) std::memcpy(angles_deg, out.angles_deg.data(), sizeof(float) * na);
    if (minmax) { minmax[0] = out.original_min_hu; minmax[1] = out.original_max_hu; }
    return 0;
}

// IReconstructionBackend::reconstructSlice (IReconstructionBackend.h:24).
// min_hu / max_hu fill Sinogram::original_min_hu / original_max_hu (OpenMP uses them).
int ref_reconstruct_slice(int which, const float* sino, int na, int nd, const float* angles_deg,
                          float min_hu, float max_hu, int n_out, int filter, float* out) {
    auto be = make_backend(which);
    Sinogram s;
    s.data.assign(static_cast<size_t>(nd), static_cast<size_t>(na));
    std::memcpy(s.data.data.data(), sino, sizeof(float) * s.data.data.size());
    s.angles_deg.assign(angles_deg, angles_deg + na);
    s.original_min_hu = min_hu;
    s.original_max_hu = max_hu;
    const Buffer2D r = be->reconstructSlice(s, static_cast<size_t>(n_out), params_for(filter, na));
    if (r.data.size() != static_cast<size_t>(n_out) * n_out) return 1;
    std::memcpy(out, r.data.data(), sizeof(float) * r.data.size());
    return 0;
}

// IReconstructionBackend::reconstructVolume (IReconstructionBackend.h:28-31);
// the reference uses detector_bins = width inside.
int ref_reconstruct_volume(int which, const float* vol, int n, int nz, int na, int filter,
                           float* out, double* sino_ms) {
    auto be = make_backend(which);
    Volume in(static_cast<size_t>(n), static_cast<size_t>(n), static_cast<size_t>(nz));
    std::memcpy(in.data.data(), vol, sizeof(float) * in.data.size());
    Volume res;
    be->reconstructVolume(in, res, params_for(filter, na), nullptr);
    if (res.data.size() != in.data.size()) return 1;
    std::memcpy(out, res.data.data(), sizeof(float) * res.data.size());
    if (sino_ms) *sino_ms = be->lastSinogramTimeMs();
    return 0;
}

// IReconstructionBackend::reconstructVolumeFromSinograms (IReconstructionBackend.h:39-44).
int ref_reconstruct_from_sinograms(int which, const float* sinos, int nz, int na, int bins,
                                   const float* angles_deg, int filter, float* out) {
    auto be = make_backend(which);
    Volume s(static_cast<size_t>(bins), static_cast<size_t>(na), static_cast<size_t>(nz));
    std::memcpy(s.data.data(), sinos, sizeof(float) * s.data.size());
    std::vector<float> ang(angles_deg, angles_deg + na);
    Volume res;
    be->reconstructVolumeFromSinograms(s, ang, res, params_for(filter, na), nullptr);
    if (res.data.size() != static_cast<size_t>(bins) * bins * nz) return 1;
    std::memcpy(out, res.data.data(), sizeof(float) * res.data.size());
    return 0;
}

// IReconstructionBackend::extractPointCloud (IReconstructionBackend.h:47); points as
// (x, y, z, hu). Returns the count through *count, writes at most cap points.
int ref_extract_point_cloud(int which, const float* vol, int nx, int ny, int nz, float thr,
                            float* pts, long long cap, long long* count) {
    auto be = make_backend(which);
    Volume v(static_cast<size_t>(nx), static_cast<size_t>(ny), static_cast<size_t>(nz));
    std::memcpy(v.data.data(), vol, sizeof(float) * v.data.size());
    const PointCloud pc = be->extractPointCloud(v, thr);
    *count = static_cast<long long>(pc.size());
    for (long long i = 0; i < *count && i < cap && pts; ++i) {
        pts[4 * i + 0] = pc[i].x; pts[4 * i + 1] = pc[i].y;
        pts[4 * i + 2] = pc[i].z; pts[4 * i + 3] = pc[i].hu;
    }
    return 0;
}

// FilterDesign::createFilter (FilterDesign.cpp:13-29): L/2+1 floats.
int ref_create_filter(int L, int filter, float* H) {
    const auto f = FilterDesign::createFilter(static_cast<size_t>(L),
                                              static_cast<ReconstructionParams::FilterType>(filter));
    std::memcpy(H, f.data(), sizeof(float) * f.size());
    return 0;
}

// Generator3DCPU::generateBrainHU (Generator3DCPU.cpp:94-117). tissue: soft then
// bone, 8 floats each {hu_min, hu_max, size_min, size_max, peripheral_only,
// r_min, r_max, probability}.
int ref_generator3d(int nx, int ny, int nz, float radius_mm, int n_ell, unsigned seed,
                    const float* tissue, float* vol) {
    Generator3D::Params p;
    p.shape = {static_cast<size_t>(nx), static_cast<size_t>(ny), static_cast<size_t>(nz)};
    p.brain_radius_mm = radius_mm;
    p.num_ellipsoids = static_cast<size_t>(n_ell);
    p.seed = seed;
    Generator3D::TissueParams* t[2] = {&p.soft_tissue, &p.bone_tissue};
    for (int i = 0; i < 2; ++i) {
        const float* q = tissue + 8 * i;
        t[i]->hu_min = q[0]; t[i]->hu_max = q[1];
        t[i]->size_min_mm = q[2]; t[i]->size_max_mm = q[3];
        t[i]->peripheral_only = q[4] != 0.0f;
        t[i]->peripheral_radius_min = q[5]; t[i]->peripheral_radius_max = q[6];
        t[i]->probability = q[7];
    }
    const Volume v = Generator3DCPU().generateBrainHU(p);
    if (v.data.size() != static_cast<size_t>(nx) * ny * nz) return 1;
    std::memcpy(vol, v.data.data(), sizeof(float) * v.data.size());
    return 0;
}

}  // extern "C"
