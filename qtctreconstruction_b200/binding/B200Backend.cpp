// B200Backend.cpp — ct::IReconstructionBackend forwarded to libctb200.so.
#include "B200Backend.h"

#include <cmath>

namespace ct {

B200Backend::B200Backend(int device) {
    if (ctb_create(&ctx_, device) != CTB_OK) ctx_ = nullptr;
}

B200Backend::~B200Backend() { ctb_destroy(ctx_); }

std::string B200Backend::name() const { return "B200 (CUDA sm_100a)"; }

bool B200Backend::isAvailable() const { return ctx_ != nullptr; }

bool B200Backend::check(ctb_status s) {
    last_status_ = s;
    last_error_ = s == CTB_OK ? "" : std::string(ctb_status_string(s)) + ": " + ctb_last_error(ctx_);
    return s == CTB_OK;
}

// SerialBackend::computeSinogram (SerialBackend.cpp:59-136): data is
// Buffer2D(width = detector_bins, height = num_angles), uniform angles
// 180/na * a, and the slice's min/max as original_min_hu / original_max_hu.
// use_parallel has no meaning on the GPU.
Sinogram B200Backend::computeSinogram(const Buffer2D& slice, size_t num_angles, size_t detector_bins,
                                      bool /*use_parallel*/) {
    Sinogram out;
    if (!ctx_ || slice.empty() || slice.width == 0 || slice.height == 0 || num_angles == 0 ||
        detector_bins == 0)
        return out;
    out.data.assign(detector_bins, num_angles);
    out.angles_deg.resize(num_angles);
    float minmax[2] = {0.0f, 0.0f};
    if (!check(ctb_compute_sinogram(ctx_, slice.data.data(), static_cast<int>(slice.width),
                                    static_cast<int>(slice.height), static_cast<int>(num_angles),
                                    static_cast<int>(detector_bins), out.data.data.data(),
                                    out.angles_deg.data(), minmax)))
        return Sinogram{};
    out.original_min_hu = minmax[0];
    out.original_max_hu = minmax[1];
    return out;
}

// SerialBackend::reconstructSlice (SerialBackend.cpp:142-255): normalised
// units, output_size x output_size. A sinogram without its own angle list
// gets the uniform one.
Buffer2D B200Backend::reconstructSlice(const Sinogram& sinogram, size_t output_size,
                                       const ReconstructionParams& params) {
    Buffer2D out;
    const size_t na = sinogram.data.height, bins = sinogram.data.width;
    if (!ctx_ || sinogram.data.empty() || na == 0 || bins == 0 || output_size == 0) return out;
    std::vector<float> uniform;
    const float* ang = sinogram.angles_deg.data();
    if (sinogram.angles_deg.size() != na) {
        uniform.resize(na);
        const float step = 180.0f / static_cast<float>(na);
        for (size_t a = 0; a < na; ++a) uniform[a] = step * static_cast<float>(a);
        ang = uniform.data();
    }
    out.assign(output_size, output_size);
    if (!check(ctb_reconstruct_slice_hu(ctx_, sinogram.data.data.data(), static_cast<int>(na),
                                        static_cast<int>(bins), ang, static_cast<int>(output_size),
                                        static_cast<int>(params.filter), sinogram.original_min_hu,
                                        sinogram.original_max_hu, out.data.data())))
        return Buffer2D{};
    return out;
}

// SerialBackend::reconstructVolume (SerialBackend.cpp:261-318): per slice,
// forward projection onto width detector bins, FBP back to width x width and
// the slice's denormalisation; coordinates are carried over; the callback
// sees every slice in order once the volume is done.
void B200Backend::reconstructVolume(const Volume& in, Volume& out, const ReconstructionParams& params,
                                    std::function<void(int, const Buffer2D&)> onSliceDone) {
    if (!ctx_ || in.empty() || in.width == 0 || in.width != in.height || in.depth == 0) return;
    out.assign(in.width, in.height, in.depth);
    out.x_coords = in.x_coords;
    out.y_coords = in.y_coords;
    out.z_coords = in.z_coords;
    if (!check(ctb_reconstruct_volume(ctx_, in.data.data(), static_cast<int>(in.width),
                                      static_cast<int>(in.depth), static_cast<int>(params.num_angles),
                                      static_cast<int>(in.width), static_cast<int>(params.filter),
                                      out.data.data()))) {
        out = Volume{};
        return;
    }
    if (onSliceDone)
        for (size_t z = 0; z < out.depth; ++z) onSliceDone(static_cast<int>(z), out.getSlice(z));
}

// The interface's default reconstructVolumeFromSinograms
// (BackendFactory.cpp:17-60): sinograms (depth, num_angles, bins) in, slices
// of bins x bins out, normalised units.
void B200Backend::reconstructVolumeFromSinograms(const Volume& sinos, const std::vector<float>& angles_deg,
                                                 Volume& out, const ReconstructionParams& params,
                                                 std::function<void(int, const Buffer2D&)> onSliceDone) {
    const size_t bins = sinos.width, na = sinos.height, depth = sinos.depth;
    if (!ctx_ || sinos.empty() || bins == 0 || na == 0 || depth == 0 || angles_deg.size() != na) return;
    out.assign(bins, bins, depth);
    if (!check(ctb_reconstruct_from_sinograms(ctx_, sinos.data.data(), static_cast<int>(depth),
                                              static_cast<int>(na), static_cast<int>(bins), angles_deg.data(),
                                              static_cast<int>(params.filter), CTB_DENORM_NONE,
                                              out.data.data()))) {
        out = Volume{};
        return;
    }
    if (onSliceDone)
        for (size_t z = 0; z < out.depth; ++z) onSliceDone(static_cast<int>(z), out.getSlice(z));
}

// SerialBackend::extractPointCloud (SerialBackend.cpp:325-346): voxels with
// hu > threshold in z, y, x order; each position from its axis's coordinate
// list when the volume has one, else the voxel index.
PointCloud B200Backend::extractPointCloud(const Volume& vol, float threshold) {
    PointCloud cloud;
    if (!ctx_ || vol.empty()) return cloud;
    int64_t count = 0;
    if (!check(ctb_extract_point_cloud(ctx_, vol.data.data(), static_cast<int>(vol.width),
                                       static_cast<int>(vol.height), static_cast<int>(vol.depth), threshold,
                                       nullptr, 0, &count)))
        return cloud;
    std::vector<float> pts(4 * static_cast<size_t>(count));
    if (count > 0 && !check(ctb_extract_point_cloud(ctx_, vol.data.data(), static_cast<int>(vol.width),
                                                    static_cast<int>(vol.height), static_cast<int>(vol.depth),
                                                    threshold, pts.data(), count, &count)))
        return cloud;
    // an axis without coordinates gives the index itself, as in the reference
    auto coord = [](const std::vector<float>& axis, float index) {
        const size_t i = static_cast<size_t>(index);
        return i < axis.size() ? axis[i] : index;
    };
    cloud.resize(static_cast<size_t>(count));
    for (int64_t i = 0; i < count; ++i) {
        const float* p = &pts[4 * static_cast<size_t>(i)];
        cloud[i] = Point{coord(vol.x_coords, p[0]), coord(vol.y_coords, p[1]), coord(vol.z_coords, p[2]), p[3]};
    }
    return cloud;
}

double B200Backend::lastSinogramTimeMs() const { return ctb_last_sinogram_ms(ctx_); }

double B200Backend::lastReconstructionTimeMs() const { return ctb_last_reconstruction_ms(ctx_); }

}  // namespace ct
