// PGM / PFM file input and output for the command-line front end.
//
// Reading follows the reference's loadPGM (src/Image.h:129-155): binary
// "P5" greylevel with a maxval of at most 255; '#' comments between header
// fields are skipped.  Writing: "P5" 8-bit images and "Pf" single-channel
// float maps (little-endian, scale -1, rows stored bottom to top as the PFM
// format defines).  Errors are returned as messages, never by exiting.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace elas_b200 {
namespace pnm {

struct Gray {
    int width = 0, height = 0;
    std::vector<uint8_t> data;   // row-major, width * height
};

namespace detail {
// next header token of a PNM file (skips whitespace and '#' comments)
inline bool token(FILE* f, std::string& out) {
    out.clear();
    int c = std::fgetc(f);
    for (;;) {
        while (c == ' ' || c == '\t' || c == '\r' || c == '\n') c = std::fgetc(f);
        if (c == '#') {
            while (c != '\n' && c != EOF) c = std::fgetc(f);
            continue;
        }
        break;
    }
    while (c != EOF && c != ' ' && c != '\t' && c != '\r' && c != '\n' && c != '#') {
        out.push_back(char(c));
        c = std::fgetc(f);
    }
    return !out.empty();   // the single whitespace after maxval has been consumed
}
inline bool parse_int(const std::string& s, int& v) {
    if (s.empty() || s.size() > 9) return false;
    v = 0;
    for (char ch : s) {
        if (ch < '0' || ch > '9') return false;
        v = v * 10 + (ch - '0');
    }
    return true;
}
}  // namespace detail

// Read a binary greylevel PGM; returns an empty string on success.
inline std::string read_pgm(const std::string& path, Gray& img) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return "cannot open " + path;
    std::string t;
    int w = 0, h = 0, maxval = 0;
    std::string err;
    if (!detail::token(f, t) || t != "P5") err = path + ": not a binary PGM (P5)";
    else if (!detail::token(f, t) || !detail::parse_int(t, w) || w <= 0) err = path + ": bad width";
    else if (!detail::token(f, t) || !detail::parse_int(t, h) || h <= 0) err = path + ": bad height";
    else if (!detail::token(f, t) || !detail::parse_int(t, maxval) || maxval <= 0 || maxval > 255)
        err = path + ": maxval must be in [1, 255]";
    if (err.empty()) {
        img.width = w;
        img.height = h;
        img.data.assign(size_t(w) * h, 0);
        if (std::fread(img.data.data(), 1, img.data.size(), f) != img.data.size()) err = path + ": truncated data";
    }
    std::fclose(f);
    return err;
}

inline std::string write_pgm(const std::string& path, const uint8_t* data, int width, int height) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return "cannot create " + path;
    std::fprintf(f, "P5\n%d %d\n255\n", width, height);
    const size_t n = size_t(width) * height;
    const bool ok = std::fwrite(data, 1, n, f) == n;
    std::fclose(f);
    return ok ? std::string() : path + ": write failed";
}

// Single-channel PFM; rows are written bottom to top.
inline std::string write_pfm(const std::string& path, const float* data, int width, int height) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return "cannot create " + path;
    std::fprintf(f, "Pf\n%d %d\n-1\n", width, height);   // negative scale: little-endian
    bool ok = true;
    for (int y = height - 1; y >= 0 && ok; --y)
        ok = std::fwrite(data + size_t(y) * width, sizeof(float), size_t(width), f) == size_t(width);
    std::fclose(f);
    return ok ? std::string() : path + ": write failed";
}

// Read a single-channel little-endian PFM written by write_pfm.
inline std::string read_pfm(const std::string& path, std::vector<float>& data, int& width, int& height) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return "cannot open " + path;
    std::string t, err;
    double scale = 0.0;
    if (!detail::token(f, t) || t != "Pf") err = path + ": not a single-channel PFM";
    else if (!detail::token(f, t) || !detail::parse_int(t, width) || width <= 0) err = path + ": bad width";
    else if (!detail::token(f, t) || !detail::parse_int(t, height) || height <= 0) err = path + ": bad height";
    else if (!detail::token(f, t) || (scale = std::atof(t.c_str())) >= 0.0) err = path + ": only little-endian PFM";
    if (err.empty()) {
        data.assign(size_t(width) * height, 0.0f);
        for (int y = height - 1; y >= 0 && err.empty(); --y)
            if (std::fread(data.data() + size_t(y) * width, sizeof(float), size_t(width), f) != size_t(width))
                err = path + ": truncated data";
    }
    std::fclose(f);
    return err;
}

// 8-bit view of a disparity map: d * 255 / disp_max, invalid (< 0) as 0.
inline std::vector<uint8_t> to_gray(const float* d, size_t n, int disp_max) {
    std::vector<uint8_t> out(n);
    const float s = disp_max > 0 ? 255.0f / float(disp_max) : 1.0f;
    for (size_t i = 0; i < n; ++i) {
        const float v = d[i] < 0 ? 0.0f : d[i] * s;
        out[i] = uint8_t(v > 255.0f ? 255.0f : v + 0.5f);
    }
    return out;
}

}  // namespace pnm
}  // namespace elas_b200
