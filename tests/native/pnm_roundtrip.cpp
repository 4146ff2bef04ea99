// PGM / PFM reading and writing of the command-line front end
// (cuda-stereo-matching_b200/cli/pnm_io.h), exercised without a GPU.
#include <cstdio>
#include <string>
#include <vector>

#include "../../cuda-stereo-matching_b200/cli/pnm_io.h"

using namespace elas_b200::pnm;

static int check(bool ok, const char* what) {
    if (!ok) std::printf("FAIL %s\n", what);
    return ok ? 0 : 1;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    int bad = 0;
    // PGM round trip
    std::vector<uint8_t> img(37 * 11);
    for (size_t i = 0; i < img.size(); ++i) img[i] = uint8_t(i * 7 + 3);
    bad += check(write_pgm(dir + "/a.pgm", img.data(), 37, 11).empty(), "write pgm");
    Gray g;
    bad += check(read_pgm(dir + "/a.pgm", g).empty() && g.width == 37 && g.height == 11 && g.data == img, "pgm round trip");
    // header with comments and a smaller maxval
    {
        FILE* f = std::fopen((dir + "/c.pgm").c_str(), "wb");
        std::fprintf(f, "P5\n# a comment\n3 # width\n2\n# maxval next\n200\n");
        const uint8_t px[6] = {1, 2, 3, 4, 5, 6};
        std::fwrite(px, 1, 6, f);
        std::fclose(f);
        Gray c;
        bad += check(read_pgm(dir + "/c.pgm", c).empty() && c.width == 3 && c.height == 2 && c.data[5] == 6,
                     "pgm with comments");
    }
    // rejected inputs
    {
        FILE* f = std::fopen((dir + "/p2.pgm").c_str(), "wb");
        std::fprintf(f, "P2\n2 2\n255\n1 2 3 4\n");
        std::fclose(f);
        Gray c;
        bad += check(!read_pgm(dir + "/p2.pgm", c).empty(), "ascii pgm rejected");
        f = std::fopen((dir + "/big.pgm").c_str(), "wb");
        std::fprintf(f, "P5\n2 2\n65535\n");
        std::fclose(f);
        bad += check(!read_pgm(dir + "/big.pgm", c).empty(), "16-bit pgm rejected");
        f = std::fopen((dir + "/short.pgm").c_str(), "wb");
        std::fprintf(f, "P5\n4 4\n255\nab");
        std::fclose(f);
        bad += check(!read_pgm(dir + "/short.pgm", c).empty(), "truncated pgm rejected");
        bad += check(!read_pgm(dir + "/missing.pgm", c).empty(), "missing file reported");
    }
    // PFM round trip, including invalid (-1) and fractional values
    std::vector<float> d(13 * 5);
    for (size_t i = 0; i < d.size(); ++i) d[i] = (i % 4 == 0) ? -1.0f : float(i) * 0.25f;
    bad += check(write_pfm(dir + "/d.pfm", d.data(), 13, 5).empty(), "write pfm");
    std::vector<float> r;
    int w = 0, h = 0;
    bad += check(read_pfm(dir + "/d.pfm", r, w, h).empty() && w == 13 && h == 5 && r == d, "pfm round trip");
    // bottom-to-top row order on disk: the first stored row is the last image row
    {
        FILE* f = std::fopen((dir + "/d.pfm").c_str(), "rb");
        char hdr[64];
        std::fgets(hdr, sizeof hdr, f);
        std::fgets(hdr, sizeof hdr, f);
        std::fgets(hdr, sizeof hdr, f);
        float first = 0;
        std::fread(&first, 4, 1, f);
        std::fclose(f);
        bad += check(first == d[size_t(4) * 13], "pfm rows bottom to top");
    }
    // 8-bit view: disp_max -> 255, invalid -> 0
    const float v[4] = {-1.0f, 0.0f, 127.5f, 255.0f};
    std::vector<uint8_t> gv = to_gray(v, 4, 255);
    bad += check(gv[0] == 0 && gv[1] == 0 && gv[2] == 128 && gv[3] == 255, "gray scaling");
    std::printf(bad ? "failures %d\n" : "ok\n", bad);
    return bad ? 1 : 0;
}
