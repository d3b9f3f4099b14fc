// sinofile.cpp — the consumer data format of the reference: a sinogram stack
// as an NPY array (depth, num_angles, bins) of little-endian float32 plus a
// sidecar "<name>.meta.json" (CtReconstructionController.cpp:1353-1482 writes
// it, :1494-1616 reads it; the NPY layout is FileIO.cpp:53-148).
//
// Reading follows the reference's rules: NPY versions 1 to 3, dtype '<f4'
// only, C order, a three-entry shape; the sidecar is optional; angles come
// from it only when their count equals num_angles (else uniform 180/na * a in
// float); min/max HU from it when both keys exist (else from the data);
// detector spacing defaults to 1 mm.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ctb200.h"

namespace {

std::string meta_path(const std::string& npy) {
    std::string p = npy;
    if (p.size() >= 4) {
        std::string tail = p.substr(p.size() - 4);
        for (char& c : tail) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
        if (tail == ".npy") p.resize(p.size() - 4);
    }
    return p + ".meta.json";
}

struct NpyHeader {
    size_t shape[3] = {0, 0, 0};
    std::streamoff data_offset = 0;
};

// Parse the NPY preamble: magic, version, header length, dict with
// 'descr': '<f4', 'fortran_order': False and a three-entry 'shape'.
bool read_header(std::ifstream& in, NpyHeader* h) {
    char magic[6] = {};
    in.read(magic, 6);
    if (!in.good() || std::memcmp(magic, "\x93NUMPY", 6) != 0) return false;
    unsigned char ver[2] = {};
    in.read(reinterpret_cast<char*>(ver), 2);
    if (!in.good()) return false;
    uint32_t hlen = 0;
    if (ver[0] == 1) {
        unsigned char b[2];
        in.read(reinterpret_cast<char*>(b), 2);
        hlen = b[0] | (b[1] << 8);
    } else if (ver[0] == 2 || ver[0] == 3) {
        unsigned char b[4];
        in.read(reinterpret_cast<char*>(b), 4);
        hlen = b[0] | (b[1] << 8) | (b[2] << 16) | (static_cast<uint32_t>(b[3]) << 24);
    } else {
        return false;
    }
    if (!in.good() || hlen == 0 || hlen > (1u << 20)) return false;
    std::string hdr(hlen, '\0');
    in.read(&hdr[0], hlen);
    if (!in.good()) return false;
    if (hdr.find("'<f4'") == std::string::npos && hdr.find("\"<f4\"") == std::string::npos) return false;
    const size_t fo = hdr.find("fortran_order");
    if (fo != std::string::npos && hdr.find("True", fo) != std::string::npos &&
        hdr.find("True", fo) < hdr.find(',', fo))
        return false;
    const size_t sk = hdr.find("shape");
    if (sk == std::string::npos) return false;
    const size_t l = hdr.find('(', sk), r = hdr.find(')', sk);
    if (l == std::string::npos || r == std::string::npos || r <= l) return false;
    std::string dims = hdr.substr(l + 1, r - l - 1);
    for (char& c : dims)
        if (c == ',') c = ' ';
    std::istringstream iss(dims);
    long long v[4] = {0, 0, 0, 0};
    int n = 0;
    while (n < 4 && (iss >> v[n])) ++n;
    if (n != 3 || v[0] <= 0 || v[1] <= 0 || v[2] <= 0) return false;
    for (int i = 0; i < 3; ++i) h->shape[i] = static_cast<size_t>(v[i]);
    h->data_offset = in.tellg();
    return true;
}

// Minimal reader of the sidecar's numeric keys: a number or an array of numbers.
bool json_number(const std::string& js, const char* key, double* out) {
    const std::string k = std::string("\"") + key + "\"";
    size_t p = js.find(k);
    if (p == std::string::npos) return false;
    p = js.find(':', p + k.size());
    if (p == std::string::npos) return false;
    const char* s = js.c_str() + p + 1;
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(s, &end);
    if (end == s || errno) return false;
    *out = v;
    return true;
}

bool json_array(const std::string& js, const char* key, std::vector<double>* out) {
    const std::string k = std::string("\"") + key + "\"";
    size_t p = js.find(k);
    if (p == std::string::npos) return false;
    p = js.find(':', p + k.size());
    if (p == std::string::npos) return false;
    p = js.find_first_not_of(" \t\r\n", p + 1);
    if (p == std::string::npos || js[p] != '[') return false;
    const size_t e = js.find(']', p);
    if (e == std::string::npos) return false;
    out->clear();
    const char* s = js.c_str() + p + 1;
    const char* stop = js.c_str() + e;
    while (s < stop) {
        while (s < stop && (*s == ',' || std::isspace(static_cast<unsigned char>(*s)))) ++s;
        if (s >= stop) break;
        char* end = nullptr;
        const double v = std::strtod(s, &end);
        if (end == s) return false;
        out->push_back(v);
        s = end;
    }
    return true;
}

}  // namespace

extern "C" {

ctb_status ctb_sinogram_file_shape(const char* path, int* depth, int* num_angles, int* bins) {
    if (!path || !depth || !num_angles || !bins) return CTB_ERR_INVALID;
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) return CTB_ERR_NOT_FOUND;
    NpyHeader h;
    if (!read_header(in, &h)) return CTB_ERR_INVALID;
    if (h.shape[0] > 0x7fffffff || h.shape[1] > 0x7fffffff || h.shape[2] > 0x7fffffff) return CTB_ERR_UNSUPPORTED;
    *depth = static_cast<int>(h.shape[0]);
    *num_angles = static_cast<int>(h.shape[1]);
    *bins = static_cast<int>(h.shape[2]);
    return CTB_OK;
}

ctb_status ctb_load_sinogram_file(const char* path, float* sinos, float* angles_deg, float* meta) {
    if (!path || !sinos) return CTB_ERR_INVALID;
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) return CTB_ERR_NOT_FOUND;
    NpyHeader h;
    if (!read_header(in, &h)) return CTB_ERR_INVALID;
    const size_t nz = h.shape[0], na = h.shape[1], bins = h.shape[2];
    const size_t count = nz * na * bins;
    in.read(reinterpret_cast<char*>(sinos), static_cast<std::streamsize>(count * sizeof(float)));
    if (!in.good()) return CTB_ERR_INVALID;
    // sidecar
    std::string js;
    {
        std::ifstream jf(meta_path(path), std::ios::binary);
        if (jf.is_open()) {
            std::ostringstream ss;
            ss << jf.rdbuf();
            js = ss.str();
        }
    }
    double spacing = 1.0, lo = 0.0, hi = 0.0;
    bool have_minmax = false;
    std::vector<double> ang;
    if (!js.empty()) {
        json_number(js, "detector_spacing_mm", &spacing);
        have_minmax = json_number(js, "original_min_hu", &lo) && json_number(js, "original_max_hu", &hi);
        json_array(js, "angles_deg", &ang);
    }
    if (angles_deg) {
        if (ang.size() == na) {
            for (size_t a = 0; a < na; ++a) angles_deg[a] = static_cast<float>(ang[a]);
        } else {
            const float step = 180.0f / static_cast<float>(na);
            for (size_t a = 0; a < na; ++a) angles_deg[a] = step * static_cast<float>(a);
        }
    }
    if (meta) {
        float mn = std::numeric_limits<float>::max(), mx = -std::numeric_limits<float>::max();
        if (have_minmax) {
            mn = static_cast<float>(lo);
            mx = static_cast<float>(hi);
        } else {
            for (size_t i = 0; i < count; ++i) {
                mn = sinos[i] < mn ? sinos[i] : mn;
                mx = sinos[i] > mx ? sinos[i] : mx;
            }
        }
        meta[0] = static_cast<float>(spacing);
        meta[1] = mn;
        meta[2] = mx;
    }
    return CTB_OK;
}

ctb_status ctb_save_sinogram_file(const char* path, const float* sinos, int depth, int num_angles, int bins,
                                  const float* angles_deg, float spacing_mm, float min_hu, float max_hu) {
    if (!path || !sinos || depth <= 0 || num_angles <= 0 || bins <= 0) return CTB_ERR_INVALID;
    std::ofstream out(path, std::ios::binary);
    if (!out.is_open()) return CTB_ERR_NOT_FOUND;
    std::ostringstream hs;
    hs << "{'descr': '<f4', 'fortran_order': False, 'shape': (" << depth << ", " << num_angles << ", " << bins
       << "), }";
    std::string hdr = hs.str();
    size_t len = hdr.size() + 1;
    while ((10 + len) % 16 != 0) ++len;
    hdr.append(len - hdr.size() - 1, ' ');
    hdr.push_back('\n');
    out.write("\x93NUMPY", 6);
    const unsigned char ver[2] = {1, 0};
    out.write(reinterpret_cast<const char*>(ver), 2);
    const unsigned char hl[2] = {static_cast<unsigned char>(hdr.size() & 0xFF),
                                 static_cast<unsigned char>(hdr.size() >> 8)};
    out.write(reinterpret_cast<const char*>(hl), 2);
    out.write(hdr.data(), static_cast<std::streamsize>(hdr.size()));
    out.write(reinterpret_cast<const char*>(sinos),
              static_cast<std::streamsize>(sizeof(float) * static_cast<size_t>(depth) * num_angles * bins));
    if (!out.good()) return CTB_ERR_INVALID;
    out.close();
    std::ofstream jf(meta_path(path), std::ios::binary);
    if (!jf.is_open()) return CTB_ERR_NOT_FOUND;
    char buf[64];
    jf << "{\n    \"version\": 1,\n    \"depth\": " << depth << ",\n    \"num_angles\": " << num_angles
       << ",\n    \"detector_bins\": " << bins << ",\n";
    std::snprintf(buf, sizeof buf, "%.9g", static_cast<double>(spacing_mm));
    jf << "    \"detector_spacing_mm\": " << buf << ",\n";
    std::snprintf(buf, sizeof buf, "%.9g", static_cast<double>(min_hu));
    jf << "    \"original_min_hu\": " << buf << ",\n";
    std::snprintf(buf, sizeof buf, "%.9g", static_cast<double>(max_hu));
    jf << "    \"original_max_hu\": " << buf << ",\n    \"angles_deg\": [";
    const float step = 180.0f / static_cast<float>(num_angles);
    for (int a = 0; a < num_angles; ++a) {
        const float v = angles_deg ? angles_deg[a] : step * static_cast<float>(a);
        std::snprintf(buf, sizeof buf, "%.9g", static_cast<double>(v));
        jf << (a ? ", " : "") << buf;
    }
    jf << "]\n}\n";
    return jf.good() ? CTB_OK : CTB_ERR_INVALID;
}

}  // extern "C"
