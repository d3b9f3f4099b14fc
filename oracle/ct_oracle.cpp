// ct_oracle.cpp — TEST INFRASTRUCTURE, not product code.
//
// A CPU restatement of QtCTReconstruction's SerialBackend path (the correctness
// oracle for the B200 backend). Only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py may load the library built from this file, and
// only as the checker; the product path never links or calls it.
//
// Two precisions:
//   * *_f32 — follows the reference's float arithmetic step by step (same order
//     of operations, same float twiddles, same libm calls) so that, compiled
//     with the same flags as the reference (-O2, no FMA contraction, no
//     fast-math), it reproduces SerialBackend bit for bit. The golden fixtures
//     under tests/golden pin this claim against the reference itself.
//   * *_f64 — the same algorithm evaluated in double precision ("FP64 rerun"):
//     exact twiddles, exact angles taken from the same float degree values, the
//     dropped-Nyquist quirk of the built-in inverse real FFT, the zero-pixel
//     skip, the integer detector centres and edge rules kept.
//
// Reference citations are paths inside the QtCTReconstruction project.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

namespace {

using cf = std::complex<float>;
using cd = std::complex<double>;
constexpr double kPiD = 3.14159265358979323846;

// Utils.cpp:44-46 — degrees to radians in float with a float pi literal.
inline float deg_to_rad_f(float deg) { return deg * 3.14159265358979323846f / 180.0f; }

// Utils.cpp:28-42 — next power of two (64-bit build).
size_t next_pow2(size_t v) {
    if (v <= 1) return 1;
    size_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

// SerialBackend.cpp:152-163 — padded detector geometry of reconstructSlice.
struct PadGeom {
    size_t sq;    // square_bins = ceil(sqrt(2) * bins)
    size_t pad;   // pad_before = sq/2 - bins/2
    size_t L;     // fft_size = max(64, nextPow2(2 * sq))
};
PadGeom pad_geom(size_t bins) {
    PadGeom g;
    g.sq = static_cast<size_t>(std::ceil(std::sqrt(2.0) * static_cast<double>(bins)));
    g.pad = g.sq / 2 - bins / 2;
    g.L = std::max<size_t>(64, next_pow2(2 * g.sq));
    return g;
}

// ---------------------------------------------------------------------------
// FP32 radix-2 FFT, following FFT.cpp:9-158 operation for operation.
// ---------------------------------------------------------------------------

// FFT.cpp:9-18 — float twiddles exp(±2*pi*i*k/n), pi rounded to 3.14159265359f.
std::vector<cf> twiddles_f32(size_t n, bool inverse) {
    std::vector<cf> tw(n / 2);
    const float step = 2.0f * 3.14159265359f / static_cast<float>(n) * (inverse ? 1.0f : -1.0f);
    for (size_t k = 0; k < n / 2; ++k) {
        const float ang = step * static_cast<float>(k);
        tw[k] = cf(std::cos(ang), std::sin(ang));
    }
    return tw;
}

// FFT.cpp:122-158 — in-place iterative decimation-in-time transform.
void fft_core_f32(std::vector<cf>& a, bool inverse) {
    const size_t n = a.size();
    if (n <= 1) return;
    // bit-reversal permutation
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    const std::vector<cf> tw = twiddles_f32(n, inverse);
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t stride = n / len;
        const size_t half = len / 2;
        for (size_t base = 0; base < n; base += len) {
            for (size_t j = 0; j < half; ++j) {
                const cf t = a[base + j + half] * tw[j * stride];
                a[base + j + half] = a[base + j] - t;
                a[base + j] += t;
            }
        }
    }
    if (inverse) {
        const float s = 1.0f / static_cast<float>(n);
        for (auto& v : a) v *= s;
    }
}

// FFT.cpp:51-85 — real forward transform through an n/2-point complex FFT.
void rfft_f32(const std::vector<float>& x, std::vector<cf>& X) {
    const size_t n = x.size();
    const size_t h = n / 2;
    std::vector<cf> z(h);
    for (size_t i = 0; i < h; ++i) z[i] = cf(x[2 * i], x[2 * i + 1]);
    fft_core_f32(z, false);
    X.assign(h + 1, cf(0.0f, 0.0f));
    const float astep = -3.14159265359f / static_cast<float>(h);
    for (size_t k = 0; k <= h / 2; ++k) {
        const size_t m = (h - k) % h;
        const cf zk = z[k];
        const cf zm = std::conj(z[m]);
        const cf ev = (zk + zm) * 0.5f;
        const cf od = (zk - zm) * cf(0, -0.5f);
        const float ang = astep * static_cast<float>(k);
        const cf w(std::cos(ang), std::sin(ang));
        X[k] = ev + w * od;
        if (k < h - k) X[h - k] = std::conj(ev - w * od);
    }
}

// FFT.cpp:87-120 — inverse real transform. The partner index of bin 0 is
// (h - 0) % h == 0, so the Nyquist bin X[h] is never read: bin 0 stands in for it.
void irfft_f32(const std::vector<cf>& X, std::vector<float>& x) {
    const size_t h = X.size() - 1;
    std::vector<cf> z(h);
    const float astep = 3.14159265359f / static_cast<float>(h);
    for (size_t k = 0; k < h; ++k) {
        const size_t m = (h - k) % h;
        const cf xk = X[k];
        const cf xm = std::conj(X[m]);
        const cf ev = (xk + xm);
        const cf od = (xk - xm) * cf(0, 1.0f);
        const float ang = astep * static_cast<float>(k);
        const cf w(std::cos(ang), std::sin(ang));
        z[k] = ev + w * od;
    }
    fft_core_f32(z, true);
    x.resize(2 * h);
    for (size_t k = 0; k < h; ++k) {
        x[2 * k] = z[k].real() * 0.5f;
        x[2 * k + 1] = z[k].imag() * 0.5f;
    }
}

// ---------------------------------------------------------------------------
// FP64 counterparts: exact twiddles, same structure (including the quirk).
// ---------------------------------------------------------------------------
void fft_core_f64(std::vector<cd>& a, bool inverse) {
    const size_t n = a.size();
    if (n <= 1) return;
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    std::vector<cd> tw(n / 2);
    const double sgn = inverse ? 1.0 : -1.0;
    for (size_t k = 0; k < n / 2; ++k) {
        const double ang = 2.0 * kPiD * static_cast<double>(k) / static_cast<double>(n);
        tw[k] = cd(std::cos(ang), sgn * std::sin(ang));
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t stride = n / len;
        const size_t half = len / 2;
        for (size_t base = 0; base < n; base += len) {
            for (size_t j = 0; j < half; ++j) {
                const cd t = a[base + j + half] * tw[j * stride];
                a[base + j + half] = a[base + j] - t;
                a[base + j] += t;
            }
        }
    }
    if (inverse) {
        const double s = 1.0 / static_cast<double>(n);
        for (auto& v : a) v *= s;
    }
}

void rfft_f64(const std::vector<double>& x, std::vector<cd>& X) {
    const size_t n = x.size();
    const size_t h = n / 2;
    std::vector<cd> z(h);
    for (size_t i = 0; i < h; ++i) z[i] = cd(x[2 * i], x[2 * i + 1]);
    fft_core_f64(z, false);
    X.assign(h + 1, cd(0.0, 0.0));
    for (size_t k = 0; k <= h / 2; ++k) {
        const size_t m = (h - k) % h;
        const cd zk = z[k];
        const cd zm = std::conj(z[m]);
        const cd ev = (zk + zm) * 0.5;
        const cd od = (zk - zm) * cd(0, -0.5);
        const double ang = -kPiD * static_cast<double>(k) / static_cast<double>(h);
        const cd w(std::cos(ang), std::sin(ang));
        X[k] = ev + w * od;
        if (k < h - k) X[h - k] = std::conj(ev - w * od);
    }
}

void irfft_f64(const std::vector<cd>& X, std::vector<double>& x) {
    const size_t h = X.size() - 1;
    std::vector<cd> z(h);
    for (size_t k = 0; k < h; ++k) {
        const size_t m = (h - k) % h;  // the dropped-Nyquist quirk, kept on purpose
        const cd xk = X[k];
        const cd xm = std::conj(X[m]);
        const cd ev = (xk + xm);
        const cd od = (xk - xm) * cd(0, 1.0);
        const double ang = kPiD * static_cast<double>(k) / static_cast<double>(h);
        const cd w(std::cos(ang), std::sin(ang));
        z[k] = ev + w * od;
    }
    fft_core_f64(z, true);
    x.resize(2 * h);
    for (size_t k = 0; k < h; ++k) {
        x[2 * k] = z[k].real() * 0.5;
        x[2 * k + 1] = z[k].imag() * 0.5;
    }
}

// Inverse real FFT that reads the Nyquist bin (the cuFFT C2R convention the
// reference's CUDA backend uses, CUDABackend.cu:636), normalised like
// irfft_f64.
void irfft_full_f64(const std::vector<cd>& X, std::vector<double>& x) {
    const size_t h = X.size() - 1;
    std::vector<cd> z(h);
    for (size_t k = 0; k < h; ++k) {
        const cd xk = X[k];
        const cd xm = std::conj(X[h - k]);
        const cd ev = (xk + xm);
        const cd od = (xk - xm) * cd(0, 1.0);
        const double ang = kPiD * static_cast<double>(k) / static_cast<double>(h);
        const cd w(std::cos(ang), std::sin(ang));
        z[k] = ev + w * od;
    }
    fft_core_f64(z, true);
    x.resize(2 * h);
    for (size_t k = 0; k < h; ++k) {
        x[2 * k] = z[k].real() * 0.5;
        x[2 * k + 1] = z[k].imag() * 0.5;
    }
}

// ---------------------------------------------------------------------------
// Filter design — FilterDesign.cpp:13-111. Filter ids follow
// ReconstructionParams::FilterType (CTTypes.h:151): Ramp, SheppLogan, Hamming,
// Cosine, Hann, Bartlett. Unknown ids fall back to Shepp-Logan like the reference.
// ---------------------------------------------------------------------------
double window_factor(int type, size_t k, size_t n, bool* applies) {
    const double freq = static_cast<double>(k) / static_cast<double>(n);
    *applies = true;
    switch (type) {
    case 0: *applies = false; return 1.0;                                   // Ramp
    case 2: return 0.54 + 0.46 * std::cos(kPiD * freq / 0.5);               // Hamming
    case 3: return std::cos(kPiD * freq);                                   // Cosine
    case 4: return 0.5 + 0.5 * std::cos(kPiD * freq / 0.5);                 // Hann
    case 5: return 1.0 - std::min(1.0, std::abs(freq) / 0.5);               // Bartlett
    default: {                                                              // Shepp-Logan
        const double om = kPiD * freq;
        if (k == 0 || !(std::abs(om) > 1e-12)) { *applies = false; return 1.0; }
        return std::sin(om) / om;
    }
    }
}

std::vector<float> filter_f32(size_t n, int type) {
    // FilterDesign.cpp:31-51 — spatial Ram-Lak kernel, float R2C, H = 2 Re, H[0] = 0.
    std::vector<float> h(n, 0.0f);
    h[0] = 0.25f;
    for (size_t i = 1; i < n; i += 2) {
        const size_t m = (i < n / 2) ? i : n - i;
        if (m == 0) continue;
        const double t = 1.0 / (kPiD * static_cast<double>(m));
        h[i] = static_cast<float>(-1.0 * t * t);
    }
    std::vector<cf> spec;
    rfft_f32(h, spec);
    const size_t ns = n / 2 + 1;
    std::vector<float> H(ns, 0.0f);
    for (size_t k = 0; k < ns; ++k) H[k] = static_cast<float>(2.0 * spec[k].real());
    H[0] = 0.0f;
    // FilterDesign.cpp:53-111 — windows applied in double, stored in float.
    // Shepp-Logan starts at k = 1; the other windows start at k = 0 (H[0] is 0 anyway).
    for (size_t k = 0; k < ns; ++k) {
        bool applies;
        const double w = window_factor(type, k, n, &applies);
        if (applies) H[k] = static_cast<float>(H[k] * w);
    }
    return H;
}

std::vector<double> filter_f64(size_t n, int type) {
    std::vector<double> h(n, 0.0);
    h[0] = 0.25;
    for (size_t i = 1; i < n; i += 2) {
        const size_t m = (i < n / 2) ? i : n - i;
        if (m == 0) continue;
        const double t = 1.0 / (kPiD * static_cast<double>(m));
        h[i] = -t * t;
    }
    std::vector<cd> spec;
    rfft_f64(h, spec);
    const size_t ns = n / 2 + 1;
    std::vector<double> H(ns, 0.0);
    for (size_t k = 0; k < ns; ++k) H[k] = 2.0 * spec[k].real();
    H[0] = 0.0;
    for (size_t k = 0; k < ns; ++k) {
        bool applies;
        const double w = window_factor(type, k, n, &applies);
        if (applies) H[k] *= w;
    }
    return H;
}

// Canonical uniform angles: SerialBackend.cpp:126-130 stores 180/na * a in float.
inline float angle_deg_f32(int a, int na) {
    return 180.0f / static_cast<float>(na) * static_cast<float>(a);
}

}  // namespace

extern "C" {

// Status: 0 ok, 1 invalid arguments (the reference returns empty buffers there).

// FilterDesign::createFilter (FilterDesign.cpp:13-29), float path. H has L/2+1 entries.
int orc_filter_f32(int L, int type, float* H) {
    if (L < 2 || (L & (L - 1)) != 0 || !H) return 1;
    const auto v = filter_f32(static_cast<size_t>(L), type);
    std::memcpy(H, v.data(), v.size() * sizeof(float));
    return 0;
}

int orc_filter_f64(int L, int type, double* H) {
    if (L < 2 || (L & (L - 1)) != 0 || !H) return 1;
    const auto v = filter_f64(static_cast<size_t>(L), type);
    std::memcpy(H, v.data(), v.size() * sizeof(double));
    return 0;
}

// Padded detector geometry used by reconstructSlice (SerialBackend.cpp:152-163).
int orc_pad_geometry(int bins, int* sq, int* pad, int* L) {
    if (bins <= 0) return 1;
    const PadGeom g = pad_geom(static_cast<size_t>(bins));
    *sq = static_cast<int>(g.sq);
    *pad = static_cast<int>(g.pad);
    *L = static_cast<int>(g.L);
    return 0;
}

// SerialBackend::computeSinogram (SerialBackend.cpp:59-136), float path.
// slice: h rows of w floats. sino: na rows of nd floats. angles_deg: na.
// minmax: {hu_min, hu_max}.
int orc_sinogram_f32(const float* slice, int w, int h, int na, int nd,
                     float* sino, float* angles_deg, float* minmax) {
    if (!slice || w <= 0 || h <= 0 || na <= 0 || nd <= 0 || !sino) return 1;
    float lo = std::numeric_limits<float>::max();
    float hi = std::numeric_limits<float>::lowest();
    const size_t npx = static_cast<size_t>(w) * h;
    for (size_t i = 0; i < npx; ++i) {
        const float v = slice[i];
        if (v < lo) lo = v;
        if (v > hi) hi = v;
    }
    float span = hi - lo;
    if (span < 1e-6f) span = 1.0f;
    const float inv_span = 1.0f / span;
    std::memset(sino, 0, sizeof(float) * static_cast<size_t>(na) * nd);
    const float cx = static_cast<float>(w - 1) * 0.5f;
    const float cy = static_cast<float>(h - 1) * 0.5f;
    const float dc = static_cast<float>(nd / 2);
    for (int a = 0; a < na; ++a) {
        const float th = deg_to_rad_f(180.0f / static_cast<float>(na) * static_cast<float>(a));
        const float c = std::cos(th);
        const float s = std::sin(th);
        float* row = sino + static_cast<size_t>(a) * nd;
        for (int y = 0; y < h; ++y) {
            const float* src = slice + static_cast<size_t>(y) * w;
            const float yy = static_cast<float>(y);
            for (int x = 0; x < w; ++x) {
                const float raw = src[x];
                if (raw == 0.0f) continue;  // background pixels are skipped (SerialBackend.cpp:104)
                const float v = (raw - lo) * inv_span;
                const float xx = static_cast<float>(x);
                const float pos = (xx - cx) * c + (yy - cy) * s + dc;
                const int i0 = static_cast<int>(std::floor(pos));
                if (i0 >= 0 && i0 < nd - 1) {
                    const float fr = pos - static_cast<float>(i0);
                    row[i0] += v * (1.0f - fr);
                    row[i0 + 1] += v * fr;
                } else if (i0 == nd - 1) {
                    row[i0] += v;
                }
            }
        }
    }
    if (angles_deg)
        for (int a = 0; a < na; ++a) angles_deg[a] = angle_deg_f32(a, na);
    if (minmax) { minmax[0] = lo; minmax[1] = hi; }
    return 0;
}

// The same forward projection in double precision. Angles are the float degree
// values of the float path, converted exactly (angles_deg == nullptr: uniform).
int orc_sinogram_f64(const float* slice, int w, int h, int na, int nd,
                     const float* angles_deg, double* sino, double* minmax) {
    if (!slice || w <= 0 || h <= 0 || na <= 0 || nd <= 0 || !sino) return 1;
    float lo_f = std::numeric_limits<float>::max();
    float hi_f = std::numeric_limits<float>::lowest();
    const size_t npx = static_cast<size_t>(w) * h;
    for (size_t i = 0; i < npx; ++i) {
        lo_f = std::min(lo_f, slice[i]);
        hi_f = std::max(hi_f, slice[i]);
    }
    const double lo = lo_f, hi = hi_f;
    double span = hi - lo;
    if (span < 1e-6) span = 1.0;
    std::memset(sino, 0, sizeof(double) * static_cast<size_t>(na) * nd);
    const double cx = (w - 1) * 0.5, cy = (h - 1) * 0.5, dc = static_cast<double>(nd / 2);
    for (int a = 0; a < na; ++a) {
        const double deg = angles_deg ? angles_deg[a] : angle_deg_f32(a, na);
        const double th = deg * kPiD / 180.0;
        const double c = std::cos(th), s = std::sin(th);
        double* row = sino + static_cast<size_t>(a) * nd;
        for (int y = 0; y < h; ++y) {
            for (int x = 0; x < w; ++x) {
                const float raw = slice[static_cast<size_t>(y) * w + x];
                if (raw == 0.0f) continue;
                const double v = (raw - lo) / span;
                const double pos = (x - cx) * c + (y - cy) * s + dc;
                const int i0 = static_cast<int>(std::floor(pos));
                if (i0 >= 0 && i0 < nd - 1) {
                    const double fr = pos - i0;
                    row[i0] += v * (1.0 - fr);
                    row[i0 + 1] += v * fr;
                } else if (i0 == nd - 1) {
                    row[i0] += v;
                }
            }
        }
    }
    if (minmax) { minmax[0] = lo; minmax[1] = hi; }
    return 0;
}

// SerialBackend::reconstructSlice (SerialBackend.cpp:142-255), float path.
// Returns normalised units like the reference (no denormalisation).
int orc_reconstruct_slice_f32(const float* sino, int na, int nd, const float* angles_deg,
                              int n_out, int filter, float* out) {
    if (!sino || na <= 0 || nd <= 0 || n_out <= 0 || !out || !angles_deg) return 1;
    const PadGeom g = pad_geom(static_cast<size_t>(nd));
    const std::vector<float> H = filter_f32(g.L, filter);
    const size_t ns = g.L / 2 + 1;
    std::vector<float> padded(g.L), q;
    std::vector<cf> spec;
    std::vector<float> filt(static_cast<size_t>(na) * g.sq);
    for (int a = 0; a < na; ++a) {
        std::fill(padded.begin(), padded.end(), 0.0f);
        const float* src = sino + static_cast<size_t>(a) * nd;
        for (int i = 0; i < nd; ++i) {
            const size_t d = i + g.pad;
            if (d < g.L) padded[d] = src[i];
        }
        rfft_f32(padded, spec);
        for (size_t k = 0; k < ns; ++k) spec[k] *= H[k];
        irfft_f32(spec, q);
        std::copy(q.begin(), q.begin() + g.sq, filt.begin() + static_cast<size_t>(a) * g.sq);
    }
    std::vector<float> ct(na), st(na);
    for (int a = 0; a < na; ++a) {
        const float th = deg_to_rad_f(angles_deg[a]);
        ct[a] = std::cos(th);
        st[a] = std::sin(th);
    }
    const float radius = static_cast<float>(n_out / 2);
    const float dc = static_cast<float>(g.sq / 2);
    const int sqi = static_cast<int>(g.sq);
    for (int y = 0; y < n_out; ++y) {
        const float yy = static_cast<float>(y) - radius;
        for (int x = 0; x < n_out; ++x) {
            const float xx = static_cast<float>(x) - radius;
            float* o = out + static_cast<size_t>(y) * n_out + x;
            if (xx * xx + yy * yy > radius * radius) { *o = 0.0f; continue; }
            float acc = 0.0f;
            for (int a = 0; a < na; ++a) {
                const float t = xx * ct[a] - yy * st[a];
                const float u = t + dc;
                const int i0 = static_cast<int>(std::floor(u));
                const int i1 = i0 + 1;
                const float fr = u - static_cast<float>(i0);
                if (i0 >= 0 && i1 < sqi) {
                    const float* f = filt.data() + static_cast<size_t>(a) * g.sq;
                    acc += f[i0] * (1.0f - fr) + f[i1] * fr;
                }
            }
            *o = acc;
        }
    }
    const float scale = 3.14159265358979323846f / (2.0f * static_cast<float>(na));
    const size_t nn = static_cast<size_t>(n_out) * n_out;
    for (size_t i = 0; i < nn; ++i) out[i] *= scale;
    return 0;
}

// Stage outputs of the float path for kernel-level checks: the filtered rows
// (na x sq, SerialBackend.cpp:174-195).
int orc_filter_rows_f32(const float* sino, int na, int nd, int filter, float* filt) {
    if (!sino || na <= 0 || nd <= 0 || !filt) return 1;
    const PadGeom g = pad_geom(static_cast<size_t>(nd));
    const std::vector<float> H = filter_f32(g.L, filter);
    const size_t ns = g.L / 2 + 1;
    std::vector<float> padded(g.L), q;
    std::vector<cf> spec;
    for (int a = 0; a < na; ++a) {
        std::fill(padded.begin(), padded.end(), 0.0f);
        for (int i = 0; i < nd; ++i) padded[i + g.pad] = sino[static_cast<size_t>(a) * nd + i];
        rfft_f32(padded, spec);
        for (size_t k = 0; k < ns; ++k) spec[k] *= H[k];
        irfft_f32(spec, q);
        std::copy(q.begin(), q.begin() + g.sq, filt + static_cast<size_t>(a) * g.sq);
    }
    return 0;
}

// The filter stage in double precision (filtered rows, na x sq).
int orc_filter_rows_f64(const double* sino, int na, int nd, int filter, double* filt) {
    if (!sino || na <= 0 || nd <= 0 || !filt) return 1;
    const PadGeom g = pad_geom(static_cast<size_t>(nd));
    const std::vector<double> H = filter_f64(g.L, filter);
    const size_t ns = g.L / 2 + 1;
    std::vector<double> padded(g.L), q;
    std::vector<cd> spec;
    for (int a = 0; a < na; ++a) {
        std::fill(padded.begin(), padded.end(), 0.0);
        for (int i = 0; i < nd; ++i) padded[i + g.pad] = sino[static_cast<size_t>(a) * nd + i];
        rfft_f64(padded, spec);
        for (size_t k = 0; k < ns; ++k) spec[k] *= H[k];
        irfft_f64(spec, q);
        std::copy(q.begin(), q.begin() + g.sq, filt + static_cast<size_t>(a) * g.sq);
    }
    return 0;
}

// Backprojection of already filtered rows (na x sq) in double precision,
// SerialBackend.cpp:197-252; scaled by pi / (2 na), normalised units.
int orc_backproject_f64(const double* filt, int na, int sq, const float* angles_deg,
                        int n_out, double* out) {
    if (!filt || na <= 0 || sq <= 0 || n_out <= 0 || !out || !angles_deg) return 1;
    std::vector<double> ct(na), st(na);
    for (int a = 0; a < na; ++a) {
        const double th = static_cast<double>(angles_deg[a]) * kPiD / 180.0;
        ct[a] = std::cos(th);
        st[a] = std::sin(th);
    }
    const double radius = static_cast<double>(n_out / 2);
    const double dc = static_cast<double>(sq / 2);
    const double scale = kPiD / (2.0 * na);
    for (int y = 0; y < n_out; ++y) {
        const double yy = y - radius;
        for (int x = 0; x < n_out; ++x) {
            const double xx = x - radius;
            double* o = out + static_cast<size_t>(y) * n_out + x;
            if (xx * xx + yy * yy > radius * radius) { *o = 0.0; continue; }
            double acc = 0.0;
            for (int a = 0; a < na; ++a) {
                const double u = xx * ct[a] - yy * st[a] + dc;
                const int i0 = static_cast<int>(std::floor(u));
                if (i0 >= 0 && i0 + 1 < sq) {
                    const double fr = u - i0;
                    const double* f = filt + static_cast<size_t>(a) * sq;
                    acc += f[i0] * (1.0 - fr) + f[i0 + 1] * fr;
                }
            }
            *o = acc * scale;
        }
    }
    return 0;
}

// reconstructSlice in double precision (normalised units).
int orc_reconstruct_slice_f64(const double* sino, int na, int nd, const float* angles_deg,
                              int n_out, int filter, double* out) {
    if (!sino || na <= 0 || nd <= 0 || n_out <= 0 || !out || !angles_deg) return 1;
    const PadGeom g = pad_geom(static_cast<size_t>(nd));
    std::vector<double> filt(static_cast<size_t>(na) * g.sq);
    orc_filter_rows_f64(sino, na, nd, filter, filt.data());
    return orc_backproject_f64(filt.data(), na, static_cast<int>(g.sq), angles_deg, n_out, out);
}

// Per-slice volume reconstruction with the reference's denormalisation
// (SerialBackend.cpp:261-318), with a caller-chosen detector count nd (the
// reference passes nd = width). vol and out: nz slices of n x n.
int orc_reconstruct_volume_f32(const float* vol, int n, int nz, int na, int nd, int filter,
                               float* out) {
    if (!vol || n <= 0 || nz <= 0 || na <= 0 || nd <= 0 || !out) return 1;
    const size_t nn = static_cast<size_t>(n) * n;
    std::vector<float> sino(static_cast<size_t>(na) * nd), ang(na);
    float mm[2];
    for (int z = 0; z < nz; ++z) {
        orc_sinogram_f32(vol + z * nn, n, n, na, nd, sino.data(), ang.data(), mm);
        float* o = out + z * nn;
        orc_reconstruct_slice_f32(sino.data(), na, nd, ang.data(), n, filter, o);
        const float span = mm[1] - mm[0];
        const float eff = (span <= 0.0f) ? 1.0f : span;
        for (size_t i = 0; i < nn; ++i) o[i] = o[i] * eff + mm[0];
    }
    return 0;
}

int orc_reconstruct_volume_f64(const float* vol, int n, int nz, int na, int nd, int filter,
                               double* out) {
    if (!vol || n <= 0 || nz <= 0 || na <= 0 || nd <= 0 || !out) return 1;
    const size_t nn = static_cast<size_t>(n) * n;
    std::vector<double> sino(static_cast<size_t>(na) * nd);
    std::vector<float> ang(na);
    for (int a = 0; a < na; ++a) ang[a] = angle_deg_f32(a, na);
    double mm[2];
    for (int z = 0; z < nz; ++z) {
        orc_sinogram_f64(vol + z * nn, n, n, na, nd, ang.data(), sino.data(), mm);
        double* o = out + z * nn;
        orc_reconstruct_slice_f64(sino.data(), na, nd, ang.data(), n, filter, o);
        const double span = mm[1] - mm[0];
        const double eff = (span <= 0.0) ? 1.0 : span;
        for (size_t i = 0; i < nn; ++i) o[i] = o[i] * eff + mm[0];
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Phantoms
// ---------------------------------------------------------------------------

// Ellipsoid records of the benchmark phantom, drawn from a seeded 64-bit
// Mersenne twister in this order per ellipsoid: centre ~ U[-0.6, 0.6]^3,
// semi-axes ~ U[0.05, 0.4]^3, a rotation as a normalised quaternion of four
// standard normals (redrawn while its squared norm is below 1e-12), density
// ~ U[-0.3, 1.0]. The draw order and distributions define the phantom, so they
// are fixed; the timed CPU baseline draws its phantom here and never loads the
// product library.
int orc_phantom_params(uint64_t seed, int count, float* out) {
    if (count < 0 || (count > 0 && !out)) return 1;
    std::mt19937_64 gen(seed);
    std::uniform_real_distribution<double> centre(-0.6, 0.6), semi(0.05, 0.4), density(-0.3, 1.0);
    std::normal_distribution<double> normal(0.0, 1.0);
    for (int e = 0; e < count; ++e) {
        double c[3], s[3], q[4];
        for (double& v : c) v = centre(gen);
        for (double& v : s) v = semi(gen);
        double norm2;
        do {
            norm2 = 0.0;
            for (double& v : q) {
                v = normal(gen);
                norm2 += v * v;
            }
        } while (norm2 < 1e-12);
        const double len = std::sqrt(norm2);
        const double w = q[0] / len, a = q[1] / len, b = q[2] / len, d = q[3] / len;
        const double rho = density(gen);
        float* r = out + 16 * e;
        r[0] = static_cast<float>(c[0]);
        r[1] = static_cast<float>(c[1]);
        r[2] = static_cast<float>(c[2]);
        // rows of the world -> body rotation of the unit quaternion (w, a, b, d)
        const double m[9] = {1 - 2 * (b * b + d * d), 2 * (a * b + w * d),     2 * (a * d - w * b),
                             2 * (a * b - w * d),     1 - 2 * (a * a + d * d), 2 * (b * d + w * a),
                             2 * (a * d + w * b),     2 * (b * d - w * a),     1 - 2 * (a * a + b * b)};
        for (int i = 0; i < 9; ++i) r[3 + i] = static_cast<float>(m[i]);
        for (int i = 0; i < 3; ++i) r[12 + i] = static_cast<float>(1.0 / (s[i] * s[i]));
        r[15] = static_cast<float>(rho);
    }
    return 0;
}

// Summed random-ellipsoid phantom (the benchmark phantom). params holds k
// records of 16 floats: centre (3), rotation rows R (9, body = R * (p - c)),
// inverse squared semi-axes (3), density (1). Voxel coordinates are
// X = (2x - (nx-1)) / nx (likewise y, z); voxels outside the unit sphere are 0.
// The arithmetic order is fixed so the device rasteriser can match it bit for bit:
// every product and sum is rounded to float separately (no fused multiply-add).
int orc_phantom_sum_slab(const float* params, int k, int nx, int ny, int nz, int z0, int nzs,
                         float* vol);
int orc_phantom_sum(const float* params, int k, int nx, int ny, int nz, float* vol) {
    return orc_phantom_sum_slab(params, k, nx, ny, nz, 0, nz, vol);
}

// A slab [z0, z0 + nzs) of the same phantom (coordinates of the full nz grid).
int orc_phantom_sum_slab(const float* params, int k, int nx, int ny, int nz, int z0, int nzs,
                         float* vol) {
    if (!params || k < 0 || nx <= 0 || ny <= 0 || nz <= 0 || z0 < 0 || nzs <= 0 ||
        z0 + nzs > nz || !vol)
        return 1;
    for (int zz = 0; zz < nzs; ++zz) {
        const int z = z0 + zz;
        const float Z = (2.0f * static_cast<float>(z) - static_cast<float>(nz - 1)) / static_cast<float>(nz);
        for (int y = 0; y < ny; ++y) {
            const float Y = (2.0f * static_cast<float>(y) - static_cast<float>(ny - 1)) / static_cast<float>(ny);
            for (int x = 0; x < nx; ++x) {
                const float X = (2.0f * static_cast<float>(x) - static_cast<float>(nx - 1)) / static_cast<float>(nx);
                float acc = 0.0f;
                const float r2 = X * X + Y * Y + Z * Z;
                if (r2 <= 1.0f) {
                    for (int e = 0; e < k; ++e) {
                        const float* p = params + 16 * e;
                        const float dx = X - p[0], dy = Y - p[1], dz = Z - p[2];
                        const float b0 = p[3] * dx + p[4] * dy + p[5] * dz;
                        const float b1 = p[6] * dx + p[7] * dy + p[8] * dz;
                        const float b2 = p[9] * dx + p[10] * dy + p[11] * dz;
                        const float q = b0 * b0 * p[12] + b1 * b1 * p[13] + b2 * b2 * p[14];
                        if (q <= 1.0f) acc += p[15];
                    }
                }
                vol[(static_cast<size_t>(zz) * ny + y) * nx + x] = acc;
            }
        }
    }
    return 0;
}

// Generator3DCPU::generateBrainHU (Generator3DCPU.cpp:35-117): axis-aligned
// ellipsoids in millimetre coordinates, max-composited over -1000 HU.
// tissue: 2 x 8 floats {hu_min, hu_max, size_min, size_max, peripheral_only,
// r_min, r_max, probability} for soft then bone tissue.
int orc_generator3d(int nx, int ny, int nz, float radius_mm, int n_ell, unsigned seed,
                    const float* tissue, float* vol) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || n_ell < 0 || !tissue || !vol) return 1;
    auto linspace = [](float a, float b, int n) {
        std::vector<float> v(n);
        if (n == 1) { v[0] = a; return v; }
        const float step = (b - a) / static_cast<float>(n - 1);
        for (int i = 0; i < n; ++i) v[i] = a + step * static_cast<float>(i);
        return v;
    };
    const auto xs = linspace(-radius_mm, radius_mm, nx);
    const auto ys = linspace(-radius_mm, radius_mm, ny);
    const auto zs = linspace(-radius_mm, radius_mm, nz);
    const size_t total = static_cast<size_t>(nx) * ny * nz;
    for (size_t i = 0; i < total; ++i) vol[i] = -1000.0f;
    std::mt19937 rng(seed);
    auto uni = [&rng](float a, float b) { std::uniform_real_distribution<float> d(a, b); return d(rng); };
    std::uniform_real_distribution<float> prob(0.0f, 1.0f);
    for (int e = 0; e < n_ell; ++e) {
        const bool bone = prob(rng) < tissue[8 + 7];
        const float* t = tissue + (bone ? 8 : 0);
        const float eff_r = std::max(0.0f, radius_mm - t[3]);
        const float theta = uni(0.0f, 6.2831853071795864769f);
        const float phi = std::acos(uni(-1.0f, 1.0f));
        float r;
        if (t[4] != 0.0f) r = uni(t[5] * eff_r, t[6] * eff_r);
        else r = eff_r * std::cbrt(uni(0.0f, 1.0f));
        const float sp = std::sin(phi);
        const float cx = r * sp * std::cos(theta);
        const float cy = r * sp * std::sin(theta);
        const float cz = r * std::cos(phi);
        const float ax = uni(t[2], t[3]);
        const float ay = uni(t[2], t[3]);
        const float az = uni(t[2], t[3]);
        const float hu = uni(t[0], t[1]);
        for (int z = 0; z < nz; ++z) {
            const float dz = zs[z] - cz;
            for (int y = 0; y < ny; ++y) {
                const float dy = ys[y] - cy;
                for (int x = 0; x < nx; ++x) {
                    const float dx = xs[x] - cx;
                    const float nrm = (dx * dx) / (ax * ax) + (dy * dy) / (ay * ay) + (dz * dz) / (az * az);
                    if (nrm <= 1.0f) {
                        float& v = vol[(static_cast<size_t>(z) * ny + y) * nx + x];
                        v = std::max(v, hu);
                    }
                }
            }
        }
    }
    return 0;
}

// SerialBackend::extractPointCloud (SerialBackend.cpp:325-346) with empty
// coordinate vectors: points are (x, y, z, hu) for hu > threshold in z, y, x
// order. Writes at most cap points; returns the total count through *count.
int orc_point_cloud(const float* vol, int nx, int ny, int nz, float thr, float* pts,
                    long long cap, long long* count) {
    if (!vol || nx <= 0 || ny <= 0 || nz <= 0 || !count) return 1;
    long long c = 0;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const float hu = vol[(static_cast<size_t>(z) * ny + y) * nx + x];
                if (hu > thr) {
                    if (pts && c < cap) {
                        float* p = pts + 4 * c;
                        p[0] = static_cast<float>(x); p[1] = static_cast<float>(y);
                        p[2] = static_cast<float>(z); p[3] = hu;
                    }
                    ++c;
                }
            }
    *count = c;
    return 0;
}


// ---------------------------------------------------------------------------
// The reference's CUDA backend conventions (CUDABackend.cu), in double
// precision: the FP64 restatement the CUDA-convention mode is checked against,
// pinned by tests/golden/cuda_conv.npz (written by the reference itself).

// CUDABackend::computeSinogram / radonForwardGatherKernel (CUDABackend.cu:
// 108-153, 524-590): every pixel normalised (v - min) / span (span < 1e-6 -> 1),
// rays through (cx + u cos, cy - u sin) with direction (sin, cos), u = bin -
// det_center, samples t = -half + i for i < floor(2 half) + 1 (half =
// sqrt(w^2 + h^2) / 2 in float), bilinear interpolation with zero outside.
int orc_cc_sinogram_f64(const float* slice, int w, int h, int na, int nd, double det_center,
                        const float* angles_deg, double* sino, float* minmax) {
    if (!slice || w <= 0 || h <= 0 || na <= 0 || nd <= 0 || !angles_deg || !sino) return 1;
    const size_t np = static_cast<size_t>(w) * h;
    float lo = slice[0], hi = slice[0];
    for (size_t i = 1; i < np; ++i) {
        lo = std::min(lo, slice[i]);
        hi = std::max(hi, slice[i]);
    }
    if (minmax) { minmax[0] = lo; minmax[1] = hi; }
    float span = hi - lo;
    if (span < 1e-6f) span = 1.0f;
    std::vector<double> v(np);
    for (size_t i = 0; i < np; ++i) v[i] = (static_cast<double>(slice[i]) - lo) / span;
    const double cx = 0.5 * (w - 1), cy = 0.5 * (h - 1);
    const float half_f = 0.5f * std::sqrt(static_cast<float>(w * w + h * h));
    const int ns = static_cast<int>(2.0f * half_f) + 1;
    auto at = [&](int x, int y) -> double {
        return (x >= 0 && x < w && y >= 0 && y < h) ? v[static_cast<size_t>(y) * w + x] : 0.0;
    };
    for (int a = 0; a < na; ++a) {
        const double th = static_cast<double>(angles_deg[a]) * kPiD / 180.0;
        const double c = std::cos(th), sn = std::sin(th);
        for (int b = 0; b < nd; ++b) {
            const double u = b - det_center;
            const double bx = cx + u * c, by = cy - u * sn;
            double sum = 0.0;
            for (int i = 0; i < ns; ++i) {
                const double t = -static_cast<double>(half_f) + i;
                const double x = bx + t * sn, y = by + t * c;
                const int x0 = static_cast<int>(std::floor(x)), y0 = static_cast<int>(std::floor(y));
                const double fx = x - x0, fy = y - y0;
                sum += (1 - fx) * (1 - fy) * at(x0, y0) + fx * (1 - fy) * at(x0 + 1, y0) +
                       (1 - fx) * fy * at(x0, y0 + 1) + fx * fy * at(x0 + 1, y0 + 1);
            }
            sino[static_cast<size_t>(a) * nd + b] = sum;
        }
    }
    return 0;
}

// CUDABackend::reconstructSlice (CUDABackend.cu:592-690): rows padded to L at
// pad_before, multiplied by H[k] for k = 0..L/2 (Nyquist kept), inverse / L,
// first sq samples; backprojection with radius (n-1)/2, detector centre
// (sq-1)/2, each tap read only when inside [0, sq), lerp v0 + (v1 - v0) frac,
// x pi / (2 na); denormalised (x span + min) when max - min > 0.
int orc_cc_reconstruct_slice_f64(const double* sino, int na, int nd, const float* angles_deg, int n_out,
                                 int filter, float min_hu, float max_hu, double* out) {
    if (!sino || na <= 0 || nd <= 0 || n_out <= 0 || !out || !angles_deg) return 1;
    const PadGeom g = pad_geom(static_cast<size_t>(nd));
    const std::vector<double> H = filter_f64(g.L, filter);
    const size_t ns = g.L / 2 + 1;
    std::vector<double> filt(static_cast<size_t>(na) * g.sq), padded(g.L), q;
    std::vector<cd> spec;
    for (int a = 0; a < na; ++a) {
        std::fill(padded.begin(), padded.end(), 0.0);
        for (int i = 0; i < nd; ++i) padded[i + g.pad] = sino[static_cast<size_t>(a) * nd + i];
        rfft_f64(padded, spec);
        for (size_t k = 0; k < ns; ++k) spec[k] *= H[k];
        irfft_full_f64(spec, q);  // normalised inverse (the C2R result x 1 / L)
        std::copy(q.begin(), q.begin() + g.sq, filt.begin() + static_cast<size_t>(a) * g.sq);
    }
    std::vector<double> ct(na), st(na);
    for (int a = 0; a < na; ++a) {
        const double th = static_cast<double>(angles_deg[a]) * kPiD / 180.0;
        ct[a] = std::cos(th);
        st[a] = std::sin(th);
    }
    const double radius = 0.5 * (n_out - 1), dc = 0.5 * (static_cast<double>(g.sq) - 1.0);
    const double scale = kPiD / (2.0 * na);
    const int sq = static_cast<int>(g.sq);
    const double span = static_cast<double>(max_hu) - static_cast<double>(min_hu);
    for (int y = 0; y < n_out; ++y) {
        const double yy = y - radius;
        for (int x = 0; x < n_out; ++x) {
            const double xx = x - radius;
            double r = 0.0;
            if (!(xx * xx + yy * yy > radius * radius)) {
                for (int a = 0; a < na; ++a) {
                    const double u = xx * ct[a] - yy * st[a] + dc;
                    const int i0 = static_cast<int>(std::floor(u));
                    const double* f = filt.data() + static_cast<size_t>(a) * sq;
                    const double v0 = (i0 >= 0 && i0 < sq) ? f[i0] : 0.0;
                    const double v1 = (i0 + 1 >= 0 && i0 + 1 < sq) ? f[i0 + 1] : 0.0;
                    r += v0 + (v1 - v0) * (u - i0);
                }
                r *= scale;
            }
            out[static_cast<size_t>(y) * n_out + x] = (max_hu - min_hu > 0.0f) ? r * span + min_hu : r;
        }
    }
    return 0;
}

// CUDABackend::reconstructVolume (CUDABackend.cu:692-...): per slice the
// forward projection onto nd = n bins with detector centre floor(n / 2), then
// reconstructSlice with the slice's own min/max.
int orc_cc_reconstruct_volume_f64(const float* vol, int n, int depth, int na, int filter, double* out) {
    if (!vol || n <= 0 || depth <= 0 || na <= 0 || !out) return 1;
    std::vector<float> ang(na);
    const float step = 180.0f / static_cast<float>(na);
    for (int a = 0; a < na; ++a) ang[a] = static_cast<float>(a) * step;
    std::vector<double> sino(static_cast<size_t>(na) * n);
    for (int z = 0; z < depth; ++z) {
        float mm[2];
        const size_t off = static_cast<size_t>(z) * n * n;
        orc_cc_sinogram_f64(vol + off, n, n, na, n, static_cast<double>(n / 2), ang.data(), sino.data(), mm);
        orc_cc_reconstruct_slice_f64(sino.data(), na, n, ang.data(), n, filter, mm[0], mm[1], out + off);
    }
    return 0;
}

}  // extern "C"
