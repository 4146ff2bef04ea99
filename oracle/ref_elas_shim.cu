// ORACLE -- test infrastructure only.
// C entry point around the reference's own GPU pipeline, Elas::process
// (src/Elas.h:76-83, src/Elas.cu:19-120): compiled from the reference tree
// (src/Elas.cu, src/Kernels/*.cu, src/triangle.cpp, unmodified) for sm_100a
// into oracle/_ref/libelasref.so by oracle/build_oracle.py.  Its kernels
// use the compile-time constants of src/Kernels/KernelsCommon.h, whatever
// the parameters, and its process() ends after the left/right check.
#include <cstdint>
#include "Elas.h"

extern "C" int ref_elas_process(const uint8_t* left, const uint8_t* right, float* disp_left, float* disp_right,
                                int width, int height) {
    if (!left || !right || !disp_left || !disp_right || width <= 0 || height <= 0) return 1;
    const int32_t dims[2] = {width, height};
    Elas elas;
    elas.process(const_cast<uint8_t*>(left), const_cast<uint8_t*>(right), disp_left, disp_right, dims);
    return 0;
}
