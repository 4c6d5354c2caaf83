"""The oracle (oracle/lattice_oracle.c) pinned against the reference ImageStack.

Golden fixtures come from the reference build itself (tests/golden/make_golden.py); when
the reference build is present, random cases are also compared live.  Everything in the
FP32 lattice is compared bit for bit: keys, vertex order, replay records, vertex values
after splat and blur, and the slice.
"""
import hashlib

import numpy as np
import pytest

import oracle
from conftest import golden
from imagestack_b200 import synth


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def assert_dump_equal(d, g):
    np.testing.assert_array_equal(d.keys, g["keys"])
    np.testing.assert_array_equal(d.replay_vtx, g["replay_vtx"])
    np.testing.assert_array_equal(d.replay_w, g["replay_w"])
    np.testing.assert_array_equal(d.splat, g["splat"])
    np.testing.assert_array_equal(d.blur, g["blur"])
    np.testing.assert_array_equal(d.out, g["out"])


@pytest.mark.parametrize("name", ["lattice_rgb_d5", "joint_gray_d3", "lattice_d16"])
def test_oracle_lattice_matches_golden(name):
    g = golden(name)
    assert_dump_equal(oracle.oracle_lattice(g["pos"], g["val"]), g)


def test_oracle_bilateral_normalisation_matches_golden():
    g = golden("lattice_rgb_d5")
    d = oracle.oracle_lattice(g["pos"], g["val"])
    img = g["image"]
    c, h, w = img.shape
    norm = (d.out[:, :c] / d.out[:, c:c + 1]).reshape(h, w, c).transpose(2, 0, 1)
    np.testing.assert_array_equal(norm, g["bilateral"])


def gt_points(img4, sigmas):
    """positions of GaussTransform::apply: channel * (1/sigma) (src/GaussTransform.cpp:177)"""
    c = img4.shape[0]
    inv = np.float32(1.0) / np.asarray(sigmas, np.float32)
    return (img4.reshape(c, -1).T * inv[None, :]).astype(np.float32)


def test_oracle_gauss_transform_reference_test_shape():
    g = golden("gt_reference_test")
    pos = gt_points(g["splat"], g["sigmas"])
    q = gt_points(g["slice"], g["sigmas"])
    val = g["values"].reshape(2, -1).T.copy()
    f, h, w = g["splat"].shape[1:]
    d = oracle.oracle_lattice(pos, val, slice_pos=q)
    np.testing.assert_array_equal(d.out.T.reshape(2, f, h, w), g["out_distinct"])
    d = oracle.oracle_lattice(pos, val)
    np.testing.assert_array_equal(d.out.T.reshape(2, f, h, w), g["out_same"])


def joint_points(im, ref, fw, fh, ft, cs):
    """JointBilateral positions for a (c, f, h, w) image with all three axes filtered."""
    c, f, h, w = im.shape
    cr = ref.shape[0]
    one = np.float32(1.0)
    pos = np.empty((f, h, w, cr + 3), np.float32)
    for k in range(cr):
        pos[..., k] = ref[k] * (one / np.float32(cs))
    pos[..., cr] = np.arange(w, dtype=np.float32)[None, None, :] * (one / np.float32(fw))
    pos[..., cr + 1] = np.arange(h, dtype=np.float32)[None, :, None] * (one / np.float32(fh))
    pos[..., cr + 2] = np.arange(f, dtype=np.float32)[:, None, None] * (one / np.float32(ft))
    val = np.concatenate([im.transpose(1, 2, 3, 0), np.ones((f, h, w, 1), np.float32)], -1)
    return pos.reshape(-1, cr + 3), val.reshape(-1, c + 1).astype(np.float32)


def test_oracle_joint_bilateral_reference_test_shape():
    g = golden("jb_reference_test")
    im, ref = g["image"], g["reference"]
    pos, val = joint_points(im, ref, g["fw"], g["fh"], g["ft"], g["cs"])
    assert pos.shape[1] == 6
    d = oracle.oracle_lattice(pos, val)
    c, f, h, w = im.shape
    norm = (d.out[:, :c] / d.out[:, c:c + 1]).reshape(f, h, w, c).transpose(3, 0, 1, 2)
    np.testing.assert_array_equal(norm, g["out"])


def test_oracle_config1_digests():
    g = golden("gt_config1_512")
    rgb = synth.image(512, 512, 3, rects=16, seed=606)
    h, w = 512, 512
    p = np.empty((h, w, 5), np.float32)
    p[:, :, 0] = np.arange(w, dtype=np.float32)[None, :] * (np.float32(1) / np.float32(8))
    p[:, :, 1] = np.arange(h, dtype=np.float32)[:, None] * (np.float32(1) / np.float32(8))
    for k in range(3):
        p[:, :, 2 + k] = rgb[k] * (np.float32(1) / np.float32(0.1))
    v = np.concatenate([rgb.transpose(1, 2, 0), np.ones((h, w, 1), np.float32)], 2)
    d = oracle.oracle_lattice(p.reshape(-1, 5), v.reshape(-1, 4).astype(np.float32))
    assert d.keys.shape[0] == int(g["vertices"])
    assert sha(d.keys) == str(g["keys_sha256"])
    assert sha(d.replay_vtx) == str(g["replay_vtx_sha256"])
    assert sha(d.replay_w) == str(g["replay_w_sha256"])
    np.testing.assert_array_equal(d.out[g["rows"]], g["out_rows"])


def test_synthetic_generator_is_pinned():
    # the fixtures depend on these exact bytes
    img = synth.image(64, 48, 3, rects=8, seed=101)
    np.testing.assert_array_equal(img, golden("lattice_rgb_d5")["image"])
    p16, _ = synth.gauss_mixture(1500, d=16, seed=505)
    np.testing.assert_array_equal(p16, golden("lattice_d16")["pos"])


def test_fp64_lattice_close_to_fp32():
    g = golden("lattice_rgb_d5")
    a = oracle.oracle_lattice(g["pos"], g["val"])
    b = oracle.oracle_lattice(g["pos"], g["val"], fp64=True)
    np.testing.assert_array_equal(a.keys, b.keys)
    np.testing.assert_allclose(b.out, a.out, rtol=1e-5, atol=1e-6)


def test_exact_gauss_transform_matches_numpy():
    rng = np.random.default_rng(3)
    p = rng.random((50, 3), dtype=np.float32) * 2
    v = rng.random((50, 2), dtype=np.float32)
    q = rng.random((7, 3), dtype=np.float32) * 2
    out = oracle.exact_gauss_transform(q, p, v)
    d2 = ((q[:, None, :].astype(np.float64) - p[None].astype(np.float64)) ** 2).sum(-1)
    ref = np.exp(-0.5 * d2) @ v.astype(np.float64)
    np.testing.assert_allclose(out, ref, rtol=1e-12)


# ---- live comparison against the reference build (skipped where it is not built) ----

needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")


def random_case(seed, n, d, vd, scale):
    rng = np.random.default_rng(seed)
    pos = (rng.standard_normal((n, d)) * scale).astype(np.float32)
    val = rng.random((n, vd), dtype=np.float32)
    return pos, val


@needs_ref
@pytest.mark.parametrize("seed,n,d,vd,scale", [
    (1, 1, 1, 1, 1.0),          # a single point, one dimension
    (2, 257, 2, 2, 3.0),
    (3, 1000, 3, 4, 5.0),
    (4, 2000, 5, 4, 10.0),
    (5, 500, 7, 3, 2.0),        # widest key that fits one 16-byte word
    (6, 500, 8, 2, 2.0),        # first multi-word key
    (7, 400, 12, 5, 1.5),
    (8, 300, 16, 8, 1.0),
    (9, 600, 5, 4, 1000.0),     # large coordinates, keys up to ~2/3 of the int16 range
])
def test_oracle_matches_reference_random(seed, n, d, vd, scale):
    pos, val = random_case(seed, n, d, vd, scale)
    a = oracle.reference_lattice(pos, val)
    b = oracle.oracle_lattice(pos, val)
    np.testing.assert_array_equal(b.keys, a.keys)
    np.testing.assert_array_equal(b.replay_vtx, a.replay_vtx)
    np.testing.assert_array_equal(b.replay_w, a.replay_w)
    np.testing.assert_array_equal(b.splat, a.splat)
    np.testing.assert_array_equal(b.blur, a.blur)
    np.testing.assert_array_equal(b.out, a.out)


def test_oracle_refuses_keys_outside_int16():
    pos = np.array([[1.0e6, 0.0, 0.0]], np.float32)
    val = np.ones((1, 2), np.float32)
    with pytest.raises(ValueError):
        oracle.oracle_lattice(pos, val)


@needs_ref
def test_oracle_matches_reference_duplicates_and_distinct_slice():
    rng = np.random.default_rng(11)
    base = (rng.standard_normal((40, 4)) * 2).astype(np.float32)
    pos = np.repeat(base, 25, axis=0)          # many identical points
    val = rng.random((1000, 3), dtype=np.float32)
    q = (rng.standard_normal((300, 4)) * 3).astype(np.float32)   # includes unseen vertices
    a = oracle.reference_lattice(pos, val, slice_pos=q)
    b = oracle.oracle_lattice(pos, val, slice_pos=q)
    np.testing.assert_array_equal(b.keys, a.keys)
    np.testing.assert_array_equal(b.out, a.out)


@needs_ref
def test_reference_operations_agree_with_oracle_lattice():
    img = synth.image(80, 60, 3, rects=6, seed=12)
    out, _ = oracle.reference_bilateral(img, 6.0, 0.15)
    pos, val = oracle.bilateral_points(img, img, 6.0, 0.15)
    d = oracle.oracle_lattice(pos, val)
    norm = (d.out[:, :3] / d.out[:, 3:4]).reshape(60, 80, 3).transpose(2, 0, 1)
    np.testing.assert_array_equal(norm, out)


@pytest.mark.parametrize("name,guide_key,sr_key,out_key", [
    ("nlmeans_d8", "guide", "sigma_p", "out"),
    ("chromablur_d3", "guide", "sigma_c", "out_permutohedral")])
def test_oracle_high_dimensional_callers(name, guide_key, sr_key, out_key):
    """NLMeans's filter (a 6-channel patch-feature guide, d = 8) and ChromaBlur's (YUV
    against its luminance, d = 3): the oracle reproduces the reference bit for bit."""
    g = golden(name)
    im = g["image"]
    pos, val = oracle.bilateral_points(im, g[guide_key], float(g["sigma_s"]), float(g[sr_key]))
    assert pos.shape[1] == g[guide_key].shape[0] + 2
    d = oracle.oracle_lattice(pos, val)
    c, h, w = im.shape
    norm = (d.out[:, :c] / d.out[:, c:c + 1]).reshape(h, w, c).transpose(2, 0, 1)
    np.testing.assert_array_equal(norm, g[out_key])


def test_oracle_nlmeans3d_shape():
    """NLMeans3D's filter (src/GaussTransform.cpp:934-941): six frames against a 6-channel
    PCA guide with frames INF share one lattice of d = 8; the oracle reproduces the
    reference's output bit for bit."""
    g = golden("nlmeans3d_d8")
    im = g["image"]
    pos, val = oracle.volume_points(im, g["guide"], float(g["sigma_s"]), float(g["sigma_p"]),
                                    float("inf"))
    assert pos.shape == (im[0].size, 8)
    d = oracle.oracle_lattice(pos, val)
    assert d.keys.shape[0] == int(g["vertices"])
    c, f, h, w = im.shape
    norm = (d.out[:, :c] / d.out[:, c:c + 1]).reshape(f, h, w, c).transpose(3, 0, 1, 2)
    np.testing.assert_array_equal(norm, g["out"])


@pytest.mark.parametrize("key,sigma_t", [("t1_5", 1.5), ("t0", 0.0), ("tinf", float("inf"))])
def test_oracle_video_frames(key, sigma_t):
    """Bilateral::apply over five frames: t as a position (d = 6), each frame alone, and the
    frames in one lattice without a t position (src/GaussTransform.cpp:532-545)."""
    g = golden("video_frames")
    im = g["image"]
    ss, sr = float(g["sigma_s"]), float(g["sigma_r"])
    c, f, h, w = im.shape
    if sigma_t == 0.0:
        frames = []
        for t in range(f):
            pos, val = oracle.bilateral_points(im[:, t], im[:, t], ss, sr)
            d = oracle.oracle_lattice(pos, val)
            frames.append((d.out[:, :c] / d.out[:, c:c + 1]).reshape(h, w, c).transpose(2, 0, 1))
        norm = np.stack(frames, 1)
    else:
        pos, val = oracle.volume_points(im, im, ss, sr, sigma_t)
        assert pos.shape[1] == (6 if sigma_t == 1.5 else 5)
        d = oracle.oracle_lattice(pos, val)
        assert d.keys.shape[0] == int(g["vertices_" + key])
        norm = (d.out[:, :c] / d.out[:, c:c + 1]).reshape(f, h, w, c).transpose(3, 0, 1, 2)
    np.testing.assert_array_equal(norm, g["out_" + key])
