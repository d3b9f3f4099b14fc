// B200Backend.h — the class a QtCTReconstruction maintainer adds to register
// the B200 backend: ct::IReconstructionBackend (IReconstructionBackend.h:10-55)
// implemented by forwarding every method to the C ABI of libctb200.so
// (include/ctb200.h). It compiles against the reference's own
// IReconstructionBackend.h and CTTypes.h; the factory branch that creates it
// (BackendFactory.cpp:62-82) is one line.
//
// Behaviour follows the interface's contract as the reference's backends
// implement it: invalid sizes give an empty result (SerialBackend.cpp:64,148),
// a device failure gives an empty result and is kept as lastError() (the
// reference's CUDA backend prints, its Hybrid backend throws), and
// isAvailable() is false without an sm_100 GPU, so that
// BackendFactory::createBestAvailable (BackendFactory.cpp:84-92) falls back.
#pragma once

#include <string>
#include <vector>

#include "IReconstructionBackend.h"
#include "ctb200.h"

namespace ct {

class B200Backend : public IReconstructionBackend {
public:
    explicit B200Backend(int device = 0);
    ~B200Backend() override;
    B200Backend(const B200Backend&) = delete;
    B200Backend& operator=(const B200Backend&) = delete;

    std::string name() const override;
    bool isAvailable() const override;
    Sinogram computeSinogram(const Buffer2D& slice, size_t num_angles, size_t detector_bins,
                             bool use_parallel = true) override;
    Buffer2D reconstructSlice(const Sinogram& sinogram, size_t output_size,
                              const ReconstructionParams& params) override;
    void reconstructVolume(const Volume& input_volume, Volume& out_reconstruction,
                           const ReconstructionParams& params,
                           std::function<void(int slice_idx, const Buffer2D& recon_slice)> onSliceDone) override;
    void reconstructVolumeFromSinograms(
        const Volume& sinograms, const std::vector<float>& angles_deg, Volume& out_reconstruction,
        const ReconstructionParams& params,
        std::function<void(int slice_idx, const Buffer2D& recon_slice)> onSliceDone) override;
    PointCloud extractPointCloud(const Volume& vol, float threshold) override;
    double lastSinogramTimeMs() const override;
    double lastReconstructionTimeMs() const override;

    // Status and message of the last failed call (CTB_OK / "" when the last
    // call succeeded).
    ctb_status lastStatus() const { return last_status_; }
    const std::string& lastError() const { return last_error_; }
    // The context, for callers that also use the C ABI's device-buffer,
    // batch or option entry points.
    ctb_ctx* context() const { return ctx_; }

private:
    bool check(ctb_status s);

    ctb_ctx* ctx_ = nullptr;
    ctb_status last_status_ = CTB_OK;
    std::string last_error_;
};

}  // namespace ct
