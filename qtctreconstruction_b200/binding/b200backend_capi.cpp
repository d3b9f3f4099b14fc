// b200backend_capi.cpp — a C entry to a ct::B200Backend object, so that
// programs without C++ (ctypes, the tests) can drive the reference-side class
// through its ct::IReconstructionBackend interface exactly as the reference's
// controller does (virtual calls on the interface, the reference's own
// Buffer2D / Volume / Sinogram containers). Shapes follow CTTypes.h:
// slices [y][x], sinograms [angle][bin], volumes [z][y][x].
#include <cstring>
#include <memory>

#include "B200Backend.h"

using ct::B200Backend;
using ct::IReconstructionBackend;

namespace {

IReconstructionBackend* be(void* h) { return static_cast<IReconstructionBackend*>(h); }

ct::ReconstructionParams params(int filter, int num_angles) {
    ct::ReconstructionParams p;
    p.filter = static_cast<ct::ReconstructionParams::FilterType>(filter);
    p.num_angles = static_cast<size_t>(num_angles);
    return p;
}

}  // namespace

extern "C" {

// Returns an IReconstructionBackend* (NULL when no backend could be made).
void* b200be_create(int device) {
    auto* b = new B200Backend(device);
    return static_cast<IReconstructionBackend*>(b);
}

void b200be_destroy(void* h) { delete be(h); }

int b200be_is_available(void* h) { return be(h)->isAvailable() ? 1 : 0; }

int b200be_name(void* h, char* buf, int cap) {
    const std::string n = be(h)->name();
    if (cap > 0) {
        std::strncpy(buf, n.c_str(), static_cast<size_t>(cap) - 1);
        buf[cap - 1] = '\0';
    }
    return static_cast<int>(n.size());
}

// Last status of the underlying B200Backend (0 = ok).
int b200be_last_status(void* h) { return static_cast<int>(static_cast<B200Backend*>(be(h))->lastStatus()); }

// computeSinogram: sino_out[na][nd], angles_out[na], minmax_out[2]; returns
// 0, or 1 when the interface returned an empty sinogram.
int b200be_compute_sinogram(void* h, const float* slice, int w, int hgt, int na, int nd, float* sino_out,
                            float* angles_out, float* minmax_out) {
    ct::Buffer2D s(static_cast<size_t>(w), static_cast<size_t>(hgt));
    std::memcpy(s.data.data(), slice, sizeof(float) * s.data.size());
    const ct::Sinogram out = be(h)->computeSinogram(s, static_cast<size_t>(na), static_cast<size_t>(nd));
    if (out.data.empty()) return 1;
    std::memcpy(sino_out, out.data.data.data(), sizeof(float) * out.data.data.size());
    std::memcpy(angles_out, out.angles_deg.data(), sizeof(float) * out.angles_deg.size());
    minmax_out[0] = out.original_min_hu;
    minmax_out[1] = out.original_max_hu;
    return 0;
}

// reconstructSlice of sino[na][nd] with angles (NULL = none given) and the
// sinogram's HU range; out[n][n].
int b200be_reconstruct_slice(void* h, const float* sino, int na, int nd, const float* angles, int n,
                             int filter, float min_hu, float max_hu, float* out) {
    ct::Sinogram s;
    s.data.assign(static_cast<size_t>(nd), static_cast<size_t>(na));
    std::memcpy(s.data.data.data(), sino, sizeof(float) * s.data.data.size());
    if (angles) s.angles_deg.assign(angles, angles + na);
    s.original_min_hu = min_hu;
    s.original_max_hu = max_hu;
    const ct::Buffer2D r = be(h)->reconstructSlice(s, static_cast<size_t>(n), params(filter, na));
    if (r.empty()) return 1;
    std::memcpy(out, r.data.data(), sizeof(float) * r.data.size());
    return 0;
}

// reconstructVolume of vol[depth][n][n]; the callback's slice indices are
// written to slices_seen (depth ints, in call order).
int b200be_reconstruct_volume(void* h, const float* vol, int n, int depth, int na, int filter, float* out,
                              int* slices_seen) {
    ct::Volume in(static_cast<size_t>(n), static_cast<size_t>(n), static_cast<size_t>(depth));
    std::memcpy(in.data.data(), vol, sizeof(float) * in.data.size());
    ct::Volume rec;
    int seen = 0;
    be(h)->reconstructVolume(in, rec, params(filter, na), [&](int z, const ct::Buffer2D& sl) {
        if (seen < depth && slices_seen) slices_seen[seen] = z;
        ++seen;
        (void)sl;
    });
    if (rec.empty() || seen != depth) return 1;
    std::memcpy(out, rec.data.data(), sizeof(float) * rec.data.size());
    return 0;
}

// reconstructVolumeFromSinograms of sinos[depth][na][bins]; out[depth][bins][bins].
int b200be_reconstruct_from_sinograms(void* h, const float* sinos, int depth, int na, int bins,
                                      const float* angles, int filter, float* out) {
    ct::Volume s(static_cast<size_t>(bins), static_cast<size_t>(na), static_cast<size_t>(depth));
    std::memcpy(s.data.data(), sinos, sizeof(float) * s.data.size());
    std::vector<float> ang(angles, angles + na);
    ct::Volume rec;
    be(h)->reconstructVolumeFromSinograms(s, ang, rec, params(filter, na), nullptr);
    if (rec.empty()) return 1;
    std::memcpy(out, rec.data.data(), sizeof(float) * rec.data.size());
    return 0;
}

// extractPointCloud: writes at most cap points (x, y, z, hu); returns the
// total count, or -1 on failure.
long long b200be_extract_point_cloud(void* h, const float* vol, int nx, int ny, int nz, float thr,
                                     float* pts, long long cap) {
    ct::Volume v(static_cast<size_t>(nx), static_cast<size_t>(ny), static_cast<size_t>(nz));
    std::memcpy(v.data.data(), vol, sizeof(float) * v.data.size());
    const ct::PointCloud c = be(h)->extractPointCloud(v, thr);
    if (static_cast<B200Backend*>(be(h))->lastStatus() != CTB_OK) return -1;
    const long long k = static_cast<long long>(c.size()) < cap ? static_cast<long long>(c.size()) : cap;
    for (long long i = 0; i < k; ++i) {
        pts[4 * i] = c[i].x;
        pts[4 * i + 1] = c[i].y;
        pts[4 * i + 2] = c[i].z;
        pts[4 * i + 3] = c[i].hu;
    }
    return static_cast<long long>(c.size());
}

double b200be_last_sinogram_ms(void* h) { return be(h)->lastSinogramTimeMs(); }
double b200be_last_reconstruction_ms(void* h) { return be(h)->lastReconstructionTimeMs(); }

}  // extern "C"
