// Headless command-line front end of the library, in place of the
// reference's demo program (src/Main.cu:66-134), whose OpenCV display is
// dropped: disparity maps are written to files instead.
//
//   elas_b200_cli LEFT.pgm RIGHT.pgm [options]   one stereo pair from PGM files
//   elas_b200_cli demo [PRESET] [options]        one seeded synthetic pair
//
// Outputs PREFIX_left.pfm / PREFIX_right.pfm (float disparities, -1 =
// invalid) and PREFIX_left.pgm / PREFIX_right.pgm (scaled so that disp_max
// maps to 255, as the reference demo describes its output).  The images
// must have the same size, as in the reference; an error is reported and
// the exit status is non-zero otherwise.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/elas_b200.h"
#include "pnm_io.h"

namespace {

void usage() {
    std::printf(
        "usage:\n"
        "  elas_b200_cli LEFT.pgm RIGHT.pgm [options]   process one stereo pair (binary greylevel PGM)\n"
        "  elas_b200_cli demo [PRESET] [options]        process one seeded synthetic pair (PRESET 0..2)\n"
        "options:\n"
        "  --out PREFIX      output prefix (default: disp)\n"
        "  --disp-max N      largest disparity (default: the parameters' value)\n"
        "  --reference       the reference kernels' constants with the post-filters off\n"
        "  --device N        CUDA device (default 0)\n"
        "  --seed S          seed of the demo pair (default 1)\n");
}

int fail(const std::string& msg) {
    std::fprintf(stderr, "ERROR: %s\n", msg.c_str());
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2 || !std::strcmp(argv[1], "-h") || !std::strcmp(argv[1], "--help")) {
        usage();
        return argc < 2 ? 1 : 0;
    }
    std::string left_path, right_path, prefix = "disp";
    bool demo = !std::strcmp(argv[1], "demo");
    int preset = 1, device = 0, disp_max = -1, a = 2;
    unsigned long long seed = 1;
    bool reference = false;
    if (demo) {
        if (a < argc && argv[a][0] != '-') preset = std::atoi(argv[a++]);
    } else {
        if (argc < 3) { usage(); return 1; }
        left_path = argv[1];
        right_path = argv[2];
        a = 3;
    }
    for (; a < argc; ++a) {
        const std::string o = argv[a];
        auto need = [&](const char* what) -> const char* {
            if (a + 1 >= argc) { std::fprintf(stderr, "ERROR: %s needs a value\n", what); std::exit(1); }
            return argv[++a];
        };
        if (o == "--out") prefix = need("--out");
        else if (o == "--disp-max") disp_max = std::atoi(need("--disp-max"));
        else if (o == "--reference") reference = true;
        else if (o == "--device") device = std::atoi(need("--device"));
        else if (o == "--seed") seed = std::strtoull(need("--seed"), nullptr, 10);
        else { usage(); return fail("unknown option " + o); }
    }

    elas_b200::pnm::Gray L, R;
    std::vector<float> gt;
    if (demo) {
        int32_t w = 0, h = 0, d = 0;
        if (elas_b200_synth_dims(preset, &w, &h, &d) != ELAS_OK) return fail("unknown demo preset");
        L.width = R.width = w;
        L.height = R.height = h;
        L.data.resize(size_t(w) * h);
        R.data.resize(L.data.size());
        gt.resize(L.data.size());
        if (elas_b200_synth_pair(preset, seed, 0, 0, 0, L.data.data(), R.data.data(), gt.data(), nullptr) != ELAS_OK)
            return fail("synthetic pair generation failed");
        if (disp_max < 0) disp_max = d;
        std::printf("Processing: synthetic pair preset %d seed %llu (%d x %d)\n", preset, seed, w, h);
    } else {
        std::string e = elas_b200::pnm::read_pgm(left_path, L);
        if (e.empty()) e = elas_b200::pnm::read_pgm(right_path, R);
        if (!e.empty()) return fail(e);
        if (L.width != R.width || L.height != R.height)
            return fail("images must be of same size, but I1: " + std::to_string(L.width) + " x " +
                        std::to_string(L.height) + ", I2: " + std::to_string(R.width) + " x " +
                        std::to_string(R.height));
        std::printf("Processing: %s, %s (%d x %d)\n", left_path.c_str(), right_path.c_str(), L.width, L.height);
    }

    elas_params p;
    if (reference) elas_params_reference(&p);
    else elas_params_default(&p);
    if (disp_max >= 0) p.disp_max = disp_max;
    elas_handle* h = nullptr;
    int rc = elas_b200_create(&p, device, &h);
    if (rc != ELAS_OK) return fail(std::string("create: ") + elas_b200_status_string(rc));
    const size_t n = size_t(L.width) * L.height;
    std::vector<float> D1(n), D2(n);
    const int32_t dims[3] = {L.width, L.height, L.width};
    auto t0 = std::chrono::steady_clock::now();
    rc = elas_b200_process(h, L.data.data(), R.data.data(), D1.data(), D2.data(), dims, nullptr);
    auto t1 = std::chrono::steady_clock::now();
    if (rc != ELAS_OK) {
        const std::string msg = elas_b200_last_error(h);
        elas_b200_destroy(h);
        return fail(std::string("process: ") + elas_b200_status_string(rc) + ": " + msg);
    }
    elas_b200_destroy(h);

    size_t valid = 0;
    for (float d : D1) valid += d >= 0;
    std::printf("  %.2f ms (first call, includes start-up), density %.3f\n",
                std::chrono::duration<double, std::milli>(t1 - t0).count(), double(valid) / double(n));
    if (!gt.empty()) {
        size_t bad = 0, cnt = 0;
        for (size_t i = 0; i < n; ++i)
            if (gt[i] > 0) {
                ++cnt;
                bad += (D1[i] < 0 || std::abs(D1[i] - gt[i]) > 2.0f);
            }
        std::printf("  bad-2px against the ground truth %.4f\n", cnt ? double(bad) / double(cnt) : 0.0);
    }
    const int scale_max = p.disp_max > 0 ? p.disp_max : 255;
    const struct { const char* tag; const std::vector<float>* d; } outs[2] = {{"left", &D1}, {"right", &D2}};
    for (const auto& o : outs) {
        const std::string base = prefix + "_" + o.tag;
        std::string e = elas_b200::pnm::write_pfm(base + ".pfm", o.d->data(), L.width, L.height);
        if (e.empty()) {
            const std::vector<uint8_t> g = elas_b200::pnm::to_gray(o.d->data(), n, scale_max);
            e = elas_b200::pnm::write_pgm(base + ".pgm", g.data(), L.width, L.height);
        }
        if (!e.empty()) return fail(e);
        std::printf("  wrote %s.pfm, %s.pgm\n", base.c_str(), base.c_str());
    }
    std::printf("... done!\n");
    return 0;
}
