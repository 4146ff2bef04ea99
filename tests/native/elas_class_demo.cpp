// The reference's call site (src/Main.cu:66-98), written against
// include/elas_b200.hpp: compiles and links unchanged.  With an argument it
// runs one synthetic pair and prints the density of D1.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "elas_b200.hpp"

int main(int argc, char** argv) {
    int32_t width = 0, height = 0, dmax = 0;
    elas_b200_synth_dims(0, &width, &height, &dmax);
    std::vector<uint8_t> I1(size_t(width) * height), I2(I1.size());
    elas_b200_synth_pair(0, 1, 0, 0, 0, I1.data(), I2.data(), nullptr, nullptr);
    const int32_t dims[2] = {width, height};
    std::vector<float> D1(I1.size()), D2(I1.size());
    if (argc < 2) return 0;
    try {
        Elas elas;
        elas.process(I1.data(), I2.data(), D1.data(), D2.data(), dims);
    } catch (const elas_b200::Error& e) {
        std::printf("error %d: %s\n", e.status, e.what());
        return 1;
    }
    size_t valid = 0;
    for (float d : D1) valid += d >= 0;
    std::printf("density %.3f\n", double(valid) / D1.size());
    return 0;
}
