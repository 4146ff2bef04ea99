// elas_b200.hpp -- header-only C++ drop-in for the reference's Elas class
// (src/Elas.h:11-83).  Same nested `parameters` struct (field order, types,
// constructor defaults of src/Elas.h:42-66) and the same
//     void process(uint8_t* I1, uint8_t* I2, float* D1, float* D2, const int32_t* dims)
// call, so an existing call site such as src/Main.cu:89-93
//     Elas elas; elas.process(I1->data, I2->data, D1_data, D2_data, dims);
// compiles unchanged against this header and libelas_b200.so.
//
// Unlike the reference (which calls exit() on CUDA errors), failures throw
// elas_b200::Error carrying the C-ABI status.
#ifndef ELAS_B200_HPP
#define ELAS_B200_HPP

#include <cstdint>
#include <stdexcept>
#include <string>

#include "elas_b200.h"

namespace elas_b200 {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& what) : std::runtime_error(what), status(s) {}
};

}  // namespace elas_b200

class Elas {
public:
    struct parameters : elas_params {
        parameters() { elas_params_default(this); }
    };
    static_assert(sizeof(parameters) == sizeof(elas_params), "parameter block must stay byte-compatible");

    explicit Elas(const parameters& p = parameters(), int device = 0) : param(p) {
        int rc = elas_b200_create(&param, device, &h_);
        if (rc != ELAS_OK) throw elas_b200::Error(rc, elas_b200_status_string(rc));
    }
    ~Elas() {
        if (h_) elas_b200_destroy(h_);
    }
    Elas(const Elas&) = delete;
    Elas& operator=(const Elas&) = delete;

    // Drop-in for Elas::process (src/Elas.h:76-83).  dims[0] = width,
    // dims[1] = height; D1/D2 receive width*height floats ((width/2)*(height/2)
    // with param.subsampling), -1 = invalid.
    void process(uint8_t* h_img0, uint8_t* h_img1, float* h_disp0, float* h_disp1, const int32_t* dims) {
        int rc = elas_b200_set_params(h_, &param);
        if (rc == ELAS_OK) rc = elas_b200_process(h_, h_img0, h_img1, h_disp0, h_disp1, dims, nullptr);
        if (rc != ELAS_OK) throw elas_b200::Error(rc, elas_b200_last_error(h_));
    }

    parameters param;

private:
    elas_handle* h_ = nullptr;
};

#endif  // ELAS_B200_HPP
