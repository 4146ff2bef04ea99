"""The C-ABI library loads without a GPU, exports every entry point that
include/elas_b200.h declares, and its parameter block matches the C layout."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import elas_b200 as eb
from conftest import REPO, gpu_available

HEADER = os.path.join(REPO, "include", "elas_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(elas_(?:b200_)?\w+)\s*\(", text)) - {"elas_params"})


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(eb.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_layout_matches_c(tmp_path):
    src = tmp_path / "layout.c"
    fields = [f for f, _ in eb.ElasParams._fields_]
    body = "\n".join(f'printf("%zu ", offsetof(elas_params, {f}));' for f in fields)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "elas_b200.h"\n'
                   f'int main(void){{ printf("%zu ", sizeof(elas_params)); {body} return 0; }}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    expect = [ctypes.sizeof(eb.ElasParams)] + [getattr(eb.ElasParams, f).offset for f in fields]
    assert out == expect


def test_parameter_presets():
    d = eb.params_default()        # reference src/Elas.h:42-66
    assert (d.disp_max, d.candidate_stepsize, d.grid_size, d.ipol_gap_width) == (255, 5, 20, 5000)
    assert abs(d.support_threshold - 0.95) < 1e-7 and d.gamma == 5 and d.sradius == 3
    r = eb.params_reference()      # reference src/Kernels/KernelsCommon.h:8-27
    assert abs(r.support_threshold - 0.85) < 1e-7 and r.gamma == 3 and r.sradius == 2
    assert r.speckle_size == 0 and r.ipol_gap_width == 0 and not r.filter_median
    c = eb.params_config(511)
    assert c.disp_max == 511 and c.speckle_size == 200 and c.ipol_gap_width == 3 and c.filter_adaptive_mean


def test_status_strings():
    lib = eb.library()
    for s in range(8):
        assert lib.elas_b200_status_string(s)


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_create_without_device_reports_no_device():
    with pytest.raises(eb.ElasError) as e:
        eb.Elas(eb.params_reference())
    assert e.value.status == 6


def test_invalid_parameters_rejected_before_device_use():
    lib = eb.library()
    h = ctypes.c_void_p()
    p = eb.params_reference()
    p.candidate_stepsize = 0
    assert lib.elas_b200_create(ctypes.byref(p), 0, ctypes.byref(h)) == 1
    p = eb.params_reference()
    p.sradius = 40
    assert lib.elas_b200_create(ctypes.byref(p), 0, ctypes.byref(h)) == 2


def test_cpp_class_header_compiles_and_links(tmp_path):
    src = os.path.join(REPO, "tests", "native", "elas_class_demo.cpp")
    exe = tmp_path / "demo"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(REPO, "include"), src, "-o", str(exe),
                    "-L", os.path.dirname(eb.LIB_PATH), "-lelas_b200",
                    "-Wl,-rpath," + os.path.dirname(eb.LIB_PATH)], check=True)
    assert exe.exists()


def test_test_mode_switch_validates_without_a_device():
    """elas_b200_set_test_mode rejects unknown flags and negative limits
    (checked on the host; a null handle is an invalid argument)."""
    lib = eb.library()
    assert lib.elas_b200_set_test_mode(None, 0, 0) == 1
