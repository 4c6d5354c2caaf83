"""The bilateral grid method (grid_gpu) against the reference's own GRID method:
JointBilateral::apply / Bilateral::apply / GaussTransform::apply with GaussTransform::GRID
(src/GaussTransform.cpp:227-290, src/DenseGrid.h).  The splat's atomics add in another
order than the reference's serial loop; everything else follows its arithmetic, so the
results agree to FP32 rounding."""
import numpy as np
import pytest

import oracle
from imagestack_b200 import synth

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def rel_err(a, b, floor_frac=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    floor = max(np.abs(b).max() * floor_frac, 1e-30)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max())


def test_grey_joint_bilateral_d3_matches_reference_grid(gpu):
    rgb = synth.image(256, 192, 3, rects=8, seed=31)
    grey = synth.luminance(rgb)
    guide = synth.luminance(synth.image(256, 192, 3, rects=8, seed=32))
    ref, _ = oracle.reference_joint_bilateral(grey, guide, 8.0, 0.1, method="grid")
    out = grey.copy()
    gpu.JointBilateral.apply(out, guide, 8.0, 8.0, 0.0, 0.1, method="grid_gpu")
    assert rel_err(out, ref) <= RTOL


def test_rgb_bilateral_d5_matches_reference_grid(gpu):
    img = synth.image(96, 64, 3, rects=6, seed=33)
    ref, _ = oracle.reference_bilateral(img, 6.0, 0.2, method="grid")
    out = img.copy()
    gpu.Bilateral.apply(out, 6.0, 6.0, 0.0, 0.2, method="grid_gpu")
    assert rel_err(out, ref) <= RTOL


def test_gauss_transform_grid_with_other_slice_positions(gpu):
    rng = np.random.default_rng(34)
    splat = rng.uniform(0, 8, (2, 1, 40, 50)).astype(np.float32)
    slice_ = rng.uniform(-1, 9, (2, 1, 40, 50)).astype(np.float32)   # other positions
    vals = np.concatenate([rng.uniform(-1, 1, (2, 1, 40, 50)),
                           np.ones((1, 1, 40, 50))]).astype(np.float32)
    sig = [1.5, 0.75]
    ref, _ = oracle.reference_gauss_transform(slice_, splat, vals, sig, method="grid")
    out = gpu.GaussTransform.apply(slice_, splat, vals, sig, method="grid_gpu")
    assert out.shape == ref.shape
    # signed values cancel: errors are measured against 1 % of the output's magnitude
    assert rel_err(out, ref, floor_frac=1e-2) <= RTOL


def test_grid_method_limits(gpu):
    img = synth.image(32, 24, 7, rects=2, seed=35)   # d = 9 positions: too many corners
    with pytest.raises(gpu.PgpuError) as e:
        gpu.Bilateral.apply(img, 4.0, 4.0, 0.0, 0.2, method="grid_gpu")
    assert e.value.code == gpu.ERR_UNSUPPORTED
