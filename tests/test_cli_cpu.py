"""Command-line front end (in place of the reference's demo program,
src/Main.cu:66-134) without a GPU: PGM / PFM input and output, argument
handling and the errors reported before any device work."""
import os
import subprocess

import numpy as np

from conftest import REPO

CLI = os.path.join(REPO, "cuda-stereo-matching_b200", "elas_b200_cli")


def test_pnm_io_roundtrip(tmp_path):
    exe = tmp_path / "pnm"
    subprocess.run(["g++", "-std=c++17", "-O1", os.path.join(REPO, "tests", "native", "pnm_roundtrip.cpp"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok"


def _pgm(path, img):
    with open(path, "wb") as f:
        f.write(b"P5\n%d %d\n255\n" % (img.shape[1], img.shape[0]))
        f.write(np.ascontiguousarray(img, np.uint8).tobytes())


def test_cli_usage_and_input_errors(tmp_path):
    assert os.path.exists(CLI), "built by build()"
    out = subprocess.run([CLI, "--help"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and "usage" in out.stdout
    out = subprocess.run([CLI], capture_output=True, text=True, timeout=60)
    assert out.returncode != 0
    a, b = tmp_path / "a.pgm", tmp_path / "b.pgm"
    _pgm(a, np.zeros((10, 12), np.uint8))
    _pgm(b, np.zeros((10, 13), np.uint8))
    out = subprocess.run([CLI, str(a), str(b)], capture_output=True, text=True, timeout=60)
    assert out.returncode != 0 and "same size" in out.stderr
    out = subprocess.run([CLI, str(a), str(tmp_path / "missing.pgm")], capture_output=True, text=True, timeout=60)
    assert out.returncode != 0 and "cannot open" in out.stderr
    out = subprocess.run([CLI, str(a), str(a), "--bogus"], capture_output=True, text=True, timeout=60)
    assert out.returncode != 0 and "unknown option" in out.stderr
