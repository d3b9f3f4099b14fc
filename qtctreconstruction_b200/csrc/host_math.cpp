// host_math.cpp — host-side numerics of libctb200: detector geometry, the
// filter responses in double precision, and phantom parameters.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <random>
#include <vector>

#include "ctb_internal.h"

namespace ctb {

namespace {
constexpr double kPi = 3.14159265358979323846;

// In-place iterative radix-2 complex FFT in double precision with exactly
// evaluated twiddles (forward sign -1).
void fft64(std::vector<std::complex<double>>& a) {
    const size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len / 2;
        for (size_t j = 0; j < half; ++j) {
            const double ang = -2.0 * kPi * static_cast<double>(j) / static_cast<double>(len);
            const std::complex<double> w(std::cos(ang), std::sin(ang));
            for (size_t b = 0; b < n; b += len) {
                const std::complex<double> t = a[b + j + half] * w;
                a[b + j + half] = a[b + j] - t;
                a[b + j] += t;
            }
        }
    }
}
}  // namespace

PadGeom pad_geometry(int bins) {
    // SerialBackend.cpp:152-163
    PadGeom g;
    g.bins = bins;
    g.sq = static_cast<int>(std::ceil(std::sqrt(2.0) * static_cast<double>(bins)));
    g.pad = g.sq / 2 - bins / 2;
    int L = 1;
    while (L < 2 * g.sq) L <<= 1;
    g.L = std::max(64, L);
    int Lc = 1;
    while (Lc < g.sq + bins - 1) Lc <<= 1;
    g.Lc = std::max(64, Lc);
    return g;
}

std::vector<double> conv_kernel(const PadGeom& g, int type, bool keep_nyquist) {
    const int L = g.L;
    const std::vector<double> H = filter_response(L, type);
    // h = IDFT_L(H~): H~ is real and even, so h = Re FFT_L(H~) / L (real, even)
    std::vector<std::complex<double>> t(L);
    for (int k = 0; k < L; ++k) t[k] = H[k <= L / 2 ? k : L - k];
    t[0] = 0.0;
    // SerialBackend's inverse FFT never reads the Nyquist bin (FFT.cpp:96); the
    // CUDA backend's cuFFT C2R does (CUDABackend.cu:636)
    if (!keep_nyquist) t[L / 2] = 0.0;
    fft64(t);
    const int dmin = -(g.pad + g.bins - 1), dmax = g.sq - 1 - g.pad;
    std::vector<double> h(dmax - dmin + 1);
    for (int d = dmin; d <= dmax; ++d) h[d - dmin] = t[((d % L) + L) % L].real() / L;
    return h;
}

std::vector<double> conv_response(const PadGeom& g, int type, bool keep_nyquist) {
    const int Lc = g.Lc;
    const std::vector<double> h = conv_kernel(g, type, keep_nyquist);
    // The device places a row's nd values at positions [0, nd) of the
    // sequence (not at pad_before), so lag d = i - pad - j is stored at
    // (d + pad) mod Lc: filtered bin i is then sequence position i.
    std::vector<std::complex<double>> hc(Lc, 0.0);
    const int dmin = -(g.pad + g.bins - 1);
    for (size_t k = 0; k < h.size(); ++k) {
        const int d = dmin + static_cast<int>(k) + g.pad;
        hc[((d % Lc) + Lc) % Lc] = h[k];
    }
    fft64(hc);
    std::vector<double> out(2 * static_cast<size_t>(Lc));
    for (int k = 0; k < Lc; ++k) {
        out[2 * k] = hc[k].real() / Lc;
        out[2 * k + 1] = hc[k].imag() / Lc;
    }
    return out;
}

std::vector<double> filter_response(int L, int type) {
    // FilterDesign.cpp:31-51: H = 2 Re DFT_L(h), h[0] = 1/4, h[odd m] = -1/(pi m)^2
    // with m folded about L/2, and H[0] = 0; windows of FilterDesign.cpp:53-111.
    std::vector<std::complex<double>> h(L, 0.0);
    h[0] = 0.25;
    for (int i = 1; i < L; i += 2) {
        const int m = (i < L / 2) ? i : L - i;
        const double t = 1.0 / (kPi * m);
        h[i] = -t * t;
    }
    fft64(h);
    std::vector<double> H(L / 2 + 1);
    for (int k = 0; k <= L / 2; ++k) H[k] = 2.0 * h[k].real();
    H[0] = 0.0;
    for (int k = 0; k <= L / 2; ++k) {
        const double f = static_cast<double>(k) / L;
        switch (type) {
        case CTB_FILTER_RAMP: break;
        case CTB_FILTER_HAMMING: H[k] *= 0.54 + 0.46 * std::cos(kPi * f / 0.5); break;
        case CTB_FILTER_COSINE: H[k] *= std::cos(kPi * f); break;
        case CTB_FILTER_HANN: H[k] *= 0.5 + 0.5 * std::cos(kPi * f / 0.5); break;
        case CTB_FILTER_BARTLETT: H[k] *= 1.0 - std::min(1.0, std::abs(f) / 0.5); break;
        default:  // Shepp-Logan (also the reference's fallback for unknown ids)
            if (k > 0) H[k] *= std::sin(kPi * f) / (kPi * f);
            break;
        }
    }
    return H;
}

// Benchmark phantom parameters: seeded 64-bit Mersenne twister; per ellipsoid
// centre U[-0.6, 0.6]^3, semi-axes U[0.05, 0.4]^3, a uniformly random rotation
// (normalised Gaussian quaternion) and density U[-0.3, 1.0].
void phantom_params(uint64_t seed, int count, float* out) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> uc(-0.6, 0.6), ua(0.05, 0.4), ud(-0.3, 1.0);
    std::normal_distribution<double> gq(0.0, 1.0);
    for (int e = 0; e < count; ++e) {
        double c[3], ax[3], q[4];
        for (double& v : c) v = uc(rng);
        for (double& v : ax) v = ua(rng);
        double nq = 0.0;
        do {
            nq = 0.0;
            for (double& v : q) { v = gq(rng); nq += v * v; }
        } while (nq < 1e-12);
        nq = std::sqrt(nq);
        for (double& v : q) v /= nq;
        const double dens = ud(rng);
        const double w = q[0], x = q[1], y = q[2], z = q[3];
        // rotation matrix of the quaternion (world = R^T body), rows of R map world -> body
        const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)},
                                {2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x)},
                                {2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)}};
        float* p = out + 16 * e;
        for (int i = 0; i < 3; ++i) p[i] = static_cast<float>(c[i]);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) p[3 + 3 * i + j] = static_cast<float>(R[i][j]);
        for (int i = 0; i < 3; ++i) p[12 + i] = static_cast<float>(1.0 / (ax[i] * ax[i]));
        p[15] = static_cast<float>(dens);
    }
}

// Conservative index-space boxes of the summed-phantom ellipsoids.
void phantom_boxes(const float* params, int count, int nx, int ny, int nz, int* boxes) {
    const int n[3] = {nx, ny, nz};
    for (int e = 0; e < count; ++e) {
        const float* p = params + 16 * e;
        for (int i = 0; i < 3; ++i) {
            // half extent along world axis i: sqrt(sum_j (R[j][i] * a_j)^2)
            double ext2 = 0.0;
            for (int j = 0; j < 3; ++j) {
                const double a = 1.0 / std::sqrt(static_cast<double>(p[12 + j]));
                const double r = p[3 + 3 * j + i];
                ext2 += r * r * a * a;
            }
            const double ext = std::sqrt(ext2) * 1.001 + 1e-6;
            // X = (2x - (n-1))/n  <=>  x = (X n + n - 1) / 2
            const double lo = ((p[i] - ext) * n[i] + n[i] - 1) / 2.0;
            const double hi = ((p[i] + ext) * n[i] + n[i] - 1) / 2.0;
            boxes[6 * e + 2 * i] = static_cast<int>(std::floor(lo)) - 2;
            boxes[6 * e + 2 * i + 1] = static_cast<int>(std::ceil(hi)) + 2;
        }
    }
}

// Generator3DCPU's random stream (Generator3DCPU.cpp:35-117, Generator3D.h:16-34):
// the same engine, distributions and draw order, so the ellipsoids are the
// reference's. ell: 7 floats {cx, cy, cz, ax, ay, az, hu} per ellipsoid.
void generator3d_params(float radius, int count, uint32_t seed, const float* tissue, float* ell) {
    std::mt19937 rng(seed);
    auto uni = [&rng](float a, float b) {
        std::uniform_real_distribution<float> d(a, b);
        return d(rng);
    };
    std::uniform_real_distribution<float> prob(0.0f, 1.0f);
    for (int e = 0; e < count; ++e) {
        const bool bone = prob(rng) < tissue[8 + 7];
        const float* t = tissue + (bone ? 8 : 0);
        const float eff = std::max(0.0f, radius - t[3]);
        const float theta = uni(0.0f, 6.2831853071795864769f);
        const float phi = std::acos(uni(-1.0f, 1.0f));
        float r;
        if (t[4] != 0.0f) r = uni(t[5] * eff, t[6] * eff);
        else r = eff * std::cbrt(uni(0.0f, 1.0f));
        const float sp = std::sin(phi);
        float* o = ell + 7 * e;
        o[0] = r * sp * std::cos(theta);
        o[1] = r * sp * std::sin(theta);
        o[2] = r * std::cos(phi);
        o[3] = uni(t[2], t[3]);
        o[4] = uni(t[2], t[3]);
        o[5] = uni(t[2], t[3]);
        o[6] = uni(t[0], t[1]);
    }
}

void generator3d_boxes(const float* ell, int count, int nx, int ny, int nz, float radius,
                       int* boxes) {
    const int n[3] = {nx, ny, nz};
    for (int e = 0; e < count; ++e) {
        const float* p = ell + 7 * e;
        for (int i = 0; i < 3; ++i) {
            if (n[i] == 1) { boxes[6 * e + 2 * i] = 0; boxes[6 * e + 2 * i + 1] = 0; continue; }
            const double step = 2.0 * radius / (n[i] - 1);
            const double lo = (p[i] - std::fabs(p[3 + i]) * 1.001 + radius) / step;
            const double hi = (p[i] + std::fabs(p[3 + i]) * 1.001 + radius) / step;
            boxes[6 * e + 2 * i] = static_cast<int>(std::floor(lo)) - 2;
            boxes[6 * e + 2 * i + 1] = static_cast<int>(std::ceil(hi)) + 2;
        }
    }
}

}  // namespace ctb

namespace ctb {

// Group the projection angles for the forward projector: angles are split by
// walked axis (|cos| >= |sin| walks rows, else columns), kept in their given
// order within each axis, and cut into groups of kFwdGroup consecutive
// angles, which walk nearly the same rows and columns and so share L1 lines.
FwdPlan forward_plan(const float* angles_deg, int na, int w, int h, int nd) {
    (void)w;
    (void)h;
    std::vector<int> lists[2];
    std::vector<double> akq(na);
    for (int a = 0; a < na; ++a) {
        // the projector's own trig (k_trig): sincospi of deg / 180 in double
        const double t = static_cast<double>(angles_deg[a]) / 180.0;
        const double c = std::fabs(std::cos(3.14159265358979323846 * t));
        const double s = std::fabs(std::sin(3.14159265358979323846 * t));
        const int axis = c >= s ? 0 : 1;
        akq[a] = axis == 0 ? c : s;
        lists[axis].push_back(a);
    }
    FwdPlan plan;
    for (int axis = 0; axis < 2; ++axis) {
        const auto& L = lists[axis];
        for (size_t i = 0; i < L.size(); i += kFwdGroup) {
            const int first = static_cast<int>(plan.order.size());
            const int cnt = static_cast<int>(std::min<size_t>(kFwdGroup, L.size() - i));
            double amin = 1.0;
            for (int k = 0; k < cnt; ++k) {
                plan.order.push_back(L[i + k]);
                amin = std::min(amin, akq[L[i + k]]);
            }
            // near 45 degrees the coefficient is 1/sqrt 2 to rounding
            const int K = std::max(1, fwd_strip_bins(std::max(amin, 0.7071)));
            plan.groups.insert(plan.groups.end(), {first, cnt, axis, K});
            plan.max_strips = std::max(plan.max_strips, (nd + K - 1) / K);
        }
    }
    return plan;
}

}  // namespace ctb
