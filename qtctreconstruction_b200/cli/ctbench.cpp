// ctbench — headless C++17 command line over the C ABI of libctb200.so
// (include/ctb200.h): the host program the reference's Qt controller would be
// for the FBP path, without a UI.
//
//   ctbench volume   [--n 512] [--slices 512] [--angles 720] [--filter 1]
//                    [--steps 10] [--warmup 3] [--filter-mode fft|tc]
//       reconstructVolume on device buffers (seeded ellipsoid phantom),
//       timed with the library's per-stage CUDA events; prints one JSON line.
//   ctbench sinofile IN.npy OUT.npy [--filter 0] [--filter-mode fft|tc]
//       the consumer path: sinograms + .meta.json in, reconstructVolumeFrom-
//       Sinograms (output size = bins, normalised units), volume NPY out.
//   ctbench serve    [--requests 32] [--rate 0] [--seed 1] [--budget-gb 64]
//                    [--copy-threads 4] [--plain]
//       a stream of uneven FBP requests from host memory (N in {64..768},
//       16..64 slices, round(pi/2 N) angles), Poisson arrivals at --rate per
//       second (0 = all at once), through the serving loop (or, with --plain,
//       one ctb_fbp call per request); prints volumes/s and p50/p99.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "ctb200.h"

namespace {

std::map<std::string, std::string> parse(int argc, char** argv, int first, std::vector<std::string>* pos) {
    std::map<std::string, std::string> kv;
    for (int i = first; i < argc; ++i) {
        std::string a = argv[i];
        if (a.rfind("--", 0) == 0) {
            const std::string k = a.substr(2);
            if (k == "plain") {
                kv[k] = "1";
            } else if (i + 1 < argc) {
                kv[k] = argv[++i];
            }
        } else {
            pos->push_back(a);
        }
    }
    return kv;
}

long long geti(const std::map<std::string, std::string>& kv, const char* k, long long def) {
    auto it = kv.find(k);
    return it == kv.end() ? def : std::atoll(it->second.c_str());
}
double getd(const std::map<std::string, std::string>& kv, const char* k, double def) {
    auto it = kv.find(k);
    return it == kv.end() ? def : std::atof(it->second.c_str());
}
int filter_mode(const std::map<std::string, std::string>& kv) {
    auto it = kv.find("filter-mode");
    return (it != kv.end() && it->second == "tc") ? CTB_FILTER_MODE_TC_BF16X3 : CTB_FILTER_MODE_FFT;
}

int odd_bins(int n) {
    int nd = static_cast<int>(std::ceil(std::sqrt(2.0) * n));
    return nd % 2 ? nd : nd + 1;
}

int die(ctb_ctx* ctx, ctb_status s, const char* what) {
    std::fprintf(stderr, "ctbench: %s: %s %s\n", what, ctb_status_string(s), ctx ? ctb_last_error(ctx) : "");
    return 1;
}

bool write_npy(const std::string& path, const float* data, int z, int y, int x) {
    std::string hdr = "{'descr': '<f4', 'fortran_order': False, 'shape': (" + std::to_string(z) + ", " +
                      std::to_string(y) + ", " + std::to_string(x) + "), }";
    size_t len = hdr.size() + 1;
    while ((10 + len) % 16 != 0) ++len;
    hdr.append(len - hdr.size() - 1, ' ');
    hdr.push_back('\n');
    std::ofstream out(path, std::ios::binary);
    if (!out.is_open()) return false;
    out.write("\x93NUMPY\x01\x00", 8);
    const unsigned char hl[2] = {static_cast<unsigned char>(hdr.size() & 0xFF), static_cast<unsigned char>(hdr.size() >> 8)};
    out.write(reinterpret_cast<const char*>(hl), 2);
    out.write(hdr.data(), static_cast<std::streamsize>(hdr.size()));
    out.write(reinterpret_cast<const char*>(data), static_cast<std::streamsize>(sizeof(float) * size_t(z) * y * x));
    return out.good();
}

int cmd_volume(const std::map<std::string, std::string>& kv) {
    const int n = static_cast<int>(geti(kv, "n", 512)), nz = static_cast<int>(geti(kv, "slices", 512));
    const int na = static_cast<int>(geti(kv, "angles", 720)), kind = static_cast<int>(geti(kv, "filter", 1));
    const int steps = static_cast<int>(geti(kv, "steps", 10)), warm = static_cast<int>(geti(kv, "warmup", 3));
    const int nd = odd_bins(n);
    ctb_ctx* ctx = nullptr;
    ctb_status s = ctb_create(&ctx, 0);
    if (s != CTB_OK) return die(nullptr, s, "create");
    ctb_set_filter_mode(ctx, filter_mode(kv));
    ctb_set_profiling(ctx, 1);  // device time per step from the library's own CUDA events
    const size_t vox = size_t(n) * n * nz;
    float *d_vol = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_vol, vox * 4) != cudaSuccess || cudaMalloc(&d_out, vox * 4) != cudaSuccess) {
        std::fprintf(stderr, "ctbench: out of device memory\n");
        return 1;
    }
    std::vector<float> params(16 * 32);
    ctb_phantom_params(2, 32, params.data());
    if ((s = ctb_phantom_sum_d(ctx, params.data(), 32, n, n, nz, d_vol)) != CTB_OK) return die(ctx, s, "phantom");
    for (int i = 0; i < warm; ++i)
        if ((s = ctb_reconstruct_volume_d(ctx, d_vol, n, nz, na, nd, kind, d_out)) != CTB_OK) return die(ctx, s, "warm-up");
    for (int i = 0; i < steps; ++i)
        if ((s = ctb_reconstruct_volume_d(ctx, d_vol, n, nz, na, nd, kind, d_out)) != CTB_OK) return die(ctx, s, "step");
    if ((s = ctb_synchronize(ctx)) != CTB_OK) return die(ctx, s, "synchronize");
    double ms = 0.0, stage[4] = {0, 0, 0, 0};
    for (int b = 0; b < steps; ++b) {
        double t[4];
        if ((s = ctb_stage_times(ctx, b, t)) != CTB_OK) return die(ctx, s, "stage times");
        for (int k = 0; k < 4; ++k) {
            stage[k] += t[k] / steps;
            ms += t[k] / steps;
        }
    }
    const double updates = double(n) * n * nz * na;
    std::printf("{\"metric\": \"FBP voxel-angle updates/s\", \"value\": %.6g, \"unit\": \"updates/s\", "
                "\"ms_per_step\": %.4f, \"stage_ms\": [%.4f, %.4f, %.4f, %.4f], \"n\": %d, \"slices\": %d, "
                "\"angles\": %d, \"detector_bins\": %d, \"filter\": %d, \"filter_mode\": \"%s\", \"steps\": %d}\n",
                updates / (ms * 1e-3), ms, stage[0], stage[1], stage[2], stage[3], n, nz, na, nd, kind,
                filter_mode(kv) == CTB_FILTER_MODE_FFT ? "fft" : "tc_bf16x3", steps);
    cudaFree(d_vol);
    cudaFree(d_out);
    ctb_destroy(ctx);
    return 0;
}

int cmd_sinofile(const std::vector<std::string>& pos, const std::map<std::string, std::string>& kv) {
    if (pos.size() < 2) {
        std::fprintf(stderr, "usage: ctbench sinofile IN.npy OUT.npy [--filter k] [--filter-mode fft|tc]\n");
        return 2;
    }
    int nz = 0, na = 0, bins = 0;
    ctb_status s = ctb_sinogram_file_shape(pos[0].c_str(), &nz, &na, &bins);
    if (s != CTB_OK) return die(nullptr, s, "read sinogram file");
    std::vector<float> sinos(size_t(nz) * na * bins), ang(na), meta(3);
    if ((s = ctb_load_sinogram_file(pos[0].c_str(), sinos.data(), ang.data(), meta.data())) != CTB_OK)
        return die(nullptr, s, "read sinogram file");
    ctb_ctx* ctx = nullptr;
    if ((s = ctb_create(&ctx, 0)) != CTB_OK) return die(nullptr, s, "create");
    ctb_set_filter_mode(ctx, filter_mode(kv));
    std::vector<float> out(size_t(nz) * bins * bins);
    const auto t0 = std::chrono::steady_clock::now();
    if ((s = ctb_reconstruct_from_sinograms(ctx, sinos.data(), nz, na, bins, ang.data(),
                                            static_cast<int>(geti(kv, "filter", 0)), CTB_DENORM_NONE,
                                            out.data())) != CTB_OK)
        return die(ctx, s, "reconstruct");
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (!write_npy(pos[1], out.data(), nz, bins, bins)) {
        std::fprintf(stderr, "ctbench: cannot write %s\n", pos[1].c_str());
        return 1;
    }
    std::printf("{\"input\": \"%s\", \"depth\": %d, \"num_angles\": %d, \"bins\": %d, \"seconds\": %.4f, "
                "\"device_ms\": %.4f, \"original_min_hu\": %.6g, \"original_max_hu\": %.6g}\n",
                pos[0].c_str(), nz, na, bins, sec, ctb_last_reconstruction_ms(ctx), meta[1], meta[2]);
    ctb_destroy(ctx);
    return 0;
}

struct Req {
    int n, nz, na, nd, filter;
    std::vector<float> sino, out;
};

int cmd_serve(const std::map<std::string, std::string>& kv) {
    const int count = static_cast<int>(geti(kv, "requests", 32));
    const double rate = getd(kv, "rate", 0.0);
    const bool plain = kv.count("plain") != 0;
    std::mt19937_64 rng(static_cast<uint64_t>(geti(kv, "seed", 1)));
    std::vector<Req> reqs(count);
    std::normal_distribution<float> nrm(0.0f, 1.0f);
    const int filters[3] = {CTB_FILTER_RAMP, CTB_FILTER_SHEPP_LOGAN, CTB_FILTER_HANN};
    for (auto& r : reqs) {
        r.n = 64 + 32 * static_cast<int>(rng() % 23);
        r.nz = 16 + static_cast<int>(rng() % 49);
        r.na = static_cast<int>(std::lround(M_PI / 2 * r.n));
        r.nd = odd_bins(r.n);
        r.filter = filters[rng() % 3];
        r.sino.resize(size_t(r.nz) * r.na * r.nd);
        for (auto& v : r.sino) v = nrm(rng);
        r.out.assign(size_t(r.nz) * r.n * r.n, 0.0f);
    }
    std::vector<double> arrive(count, 0.0);
    if (rate > 0) {
        std::exponential_distribution<double> ex(rate);
        for (int i = 1; i < count; ++i) arrive[i] = arrive[i - 1] + ex(rng);
    }
    using Clock = std::chrono::steady_clock;
    std::vector<double> lat(count);
    double span = 0.0;
    if (plain) {
        ctb_ctx* ctx = nullptr;
        ctb_status s = ctb_create(&ctx, 0);
        if (s != CTB_OK) return die(nullptr, s, "create");
        const auto t0 = Clock::now();
        for (int i = 0; i < count; ++i) {
            const double now = std::chrono::duration<double>(Clock::now() - t0).count();
            if (now < arrive[i]) std::this_thread::sleep_for(std::chrono::duration<double>(arrive[i] - now));
            Req& r = reqs[i];
            if ((s = ctb_fbp(ctx, r.sino.data(), r.nz, r.na, r.nd, nullptr, r.n, r.filter, r.out.data())) != CTB_OK)
                return die(ctx, s, "fbp");
            lat[i] = (std::chrono::duration<double>(Clock::now() - t0).count() - arrive[i]) * 1e3;
        }
        span = std::chrono::duration<double>(Clock::now() - t0).count();
        ctb_destroy(ctx);
    } else {
        ctb_server_config cfg{};
        cfg.memory_budget = static_cast<size_t>(getd(kv, "budget-gb", 64.0) * (1ull << 30));
        cfg.copy_threads = static_cast<int>(geti(kv, "copy-threads", 4));
        ctb_server* srv = nullptr;
        ctb_status s = ctb_server_create(&cfg, &srv);
        if (s != CTB_OK) return die(nullptr, s, "server");
        std::vector<uint64_t> ids(count);
        const auto t0 = Clock::now();
        for (int i = 0; i < count; ++i) {
            const double now = std::chrono::duration<double>(Clock::now() - t0).count();
            if (now < arrive[i]) std::this_thread::sleep_for(std::chrono::duration<double>(arrive[i] - now));
            Req& r = reqs[i];
            ctb_request q{};
            q.sino = r.sino.data();
            q.depth = r.nz;
            q.num_angles = r.na;
            q.bins = r.nd;
            q.output_size = r.n;
            q.filter = r.filter;
            q.out = r.out.data();
            if ((s = ctb_server_submit(srv, &q, &ids[i])) != CTB_OK) return die(nullptr, s, "submit");
        }
        for (int i = 0; i < count; ++i)
            if ((s = ctb_server_wait(srv, ids[i], -1.0)) != CTB_OK) return die(nullptr, s, "request");
        span = std::chrono::duration<double>(Clock::now() - t0).count();
        ctb_server_stats st{};
        ctb_server_get_stats(srv, &st);
        std::printf("{\"mode\": \"served\", \"requests\": %d, \"rate_per_s\": %.4g, \"volumes_per_s\": %.4f, "
                    "\"p50_ms\": %.3f, \"p99_ms\": %.3f, \"batches\": %llu, \"mean_batch\": %.3f, "
                    "\"memory_peak\": %zu}\n",
                    count, rate, st.volumes_per_s, st.p50_ms, st.p99_ms,
                    static_cast<unsigned long long>(st.batches), st.mean_batch, st.memory_peak);
        ctb_server_destroy(srv);
        return 0;
    }
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double p) { return lat[std::min<size_t>(lat.size() - 1, size_t(std::ceil(p * lat.size())) - 1)]; };
    std::printf("{\"mode\": \"plain\", \"requests\": %d, \"rate_per_s\": %.4g, \"volumes_per_s\": %.4f, "
                "\"p50_ms\": %.3f, \"p99_ms\": %.3f}\n",
                count, rate, count / span, pct(0.5), pct(0.99));
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ctbench volume|sinofile|serve [options]\n");
        return 2;
    }
    std::vector<std::string> pos;
    const auto kv = parse(argc, argv, 2, &pos);
    const std::string cmd = argv[1];
    if (cmd == "volume") return cmd_volume(kv);
    if (cmd == "sinofile") return cmd_sinofile(pos, kv);
    if (cmd == "serve") return cmd_serve(kv);
    std::fprintf(stderr, "usage: ctbench volume|sinofile|serve [options]\n");
    return 2;
}
