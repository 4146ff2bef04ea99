// ORACLE -- test infrastructure only.
// C entry point around the reference's own Triangle (src/triangle.cpp,
// namespace TRILIB), called exactly as Elas::computeDelaunyTrianguation
// does (src/Elas.cu:282-328): float point list, switches "zQB".  Compiled
// together with the reference's triangle.cpp, from the reference tree, into
// oracle/_ref/libreftriangle.so by oracle/build_oracle.py.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include "triangle.h"

extern "C" int ref_triangulate(const float* xy, int n, int32_t* tris, int cap) {
    if (n < 3) return 0;   // Triangle exits the process below three vertices
    TRILIB::triangulateio in, out;
    std::memset(&in, 0, sizeof(in));
    std::memset(&out, 0, sizeof(out));
    in.numberofpoints = n;
    in.pointlist = (float*)std::malloc(sizeof(float) * 2 * size_t(n));
    std::memcpy(in.pointlist, xy, sizeof(float) * 2 * size_t(n));
    char sw[] = "zQB";
    TRILIB::triangulate(sw, &in, &out, nullptr);
    int nt = out.numberoftriangles;
    if (tris && nt <= cap) std::memcpy(tris, out.trianglelist, sizeof(int32_t) * 3 * size_t(nt));
    std::free(in.pointlist);
    std::free(out.pointlist);
    std::free(out.trianglelist);
    return nt;
}
