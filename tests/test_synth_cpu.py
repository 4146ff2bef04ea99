"""Seeded synthetic stereo scenes."""
import numpy as np
import pytest

import elas_b200 as eb


@pytest.mark.parametrize("preset", [0, 1, 3])
def test_synth_deterministic_and_in_range(preset):
    W, H, D = eb.synth_dims(preset)
    a = eb.synth_pair(preset, 42)
    b = eb.synth_pair(preset, 42)
    c = eb.synth_pair(preset, 43)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert not np.array_equal(a[0], c[0])
    L, R, gl, gr = a
    assert L.shape == (H, W) and R.shape == (H, W)
    assert gl.min() > 0 and gl.max() < D and gr.min() > 0 and gr.max() < D
    assert 100 < L.mean() < 156 and 20 < L.std() < 60


def test_synth_right_view_is_the_warped_left_view():
    L, R, gl, _ = eb.synth_pair(0, 3)
    H, W = L.shape
    v, u = np.mgrid[0:H, 0:W]
    ur = np.round(u - gl).astype(int)
    ok = (ur >= 0) & (ur < W)
    diff = np.abs(L[ok].astype(int) - R[v[ok], ur[ok]].astype(int))
    assert np.median(diff) < 8


def test_synth_custom_size():
    L, R, gl, gr = eb.synth_pair(3, 1, width=320, height=240, disp_max=64)
    assert L.shape == (240, 320) and gl.max() < 64


@pytest.mark.parametrize("preset,seed", [(0, 5), (1, 1000), (3, 12)])
def test_oracle_carries_the_same_generator_and_presets(preset, seed):
    """The benchmark's CPU baseline and reference arm take their inputs and
    parameters from the oracle library, so they load no product library:
    the oracle's copies must equal the library's."""
    import oracle

    kw = dict(width=320, height=240, disp_max=64) if preset == 3 else {}
    a = eb.synth_pair(preset, seed, **kw)
    b = oracle.synth_pair(preset, seed, **kw)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert oracle.synth_dims(preset) == eb.synth_dims(preset)
    assert oracle.params_reference().as_dict() == eb.params_reference().as_dict()
    for D in (63, 255, 511):
        for post in (True, False):
            assert oracle.params_config(D, post).as_dict() == eb.params_config(D, post).as_dict()
