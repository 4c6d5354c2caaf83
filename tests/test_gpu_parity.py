"""Parity of the CUDA lattice (through the C ABI) with the reference ImageStack.

Bit-exact: lattice keys, the occupied-vertex set in the reference's vertex order, the
per-point vertex indices and barycentric weights.  Within 1e-5 relative (FP32 payload):
vertex values after splat and blur and the filtered outputs; the splat's atomics sum in
a different order than the reference's serial loop, so only these may differ.
"""
import hashlib

import numpy as np
import pytest

import oracle
from conftest import golden
from imagestack_b200 import synth

pytestmark = pytest.mark.gpu

RTOL_FP32 = 1e-5


def rel_err(a, b, floor_frac=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    floor = max(np.abs(b).max() * floor_frac, 1e-30)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max()) if b.size else 0.0


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def check_dump(d, g, rtol=RTOL_FP32):
    np.testing.assert_array_equal(d["keys"], g["keys"])
    np.testing.assert_array_equal(d["replay_vtx"], g["replay_vtx"])
    np.testing.assert_array_equal(d["replay_w"], g["replay_w"])
    assert rel_err(d["splat"], g["splat"]) <= rtol
    assert rel_err(d["blur"], g["blur"]) <= rtol
    assert rel_err(d["out"], g["out"]) <= rtol


@pytest.mark.parametrize("name", ["lattice_rgb_d5", "joint_gray_d3", "lattice_d16"])
def test_lattice_dump_matches_reference(gpu, name):
    g = golden(name)
    check_dump(gpu.lattice_dump(g["pos"], g["val"]), g)


def test_bilateral_matches_reference(gpu):
    g = golden("lattice_rgb_d5")
    img = g["image"].copy()
    gpu.Bilateral.apply(img, float(g["sigma_s"]), float(g["sigma_s"]), 0.0, float(g["sigma_r"]))
    assert rel_err(img, g["bilateral"]) <= RTOL_FP32


def test_joint_bilateral_gray_d3_matches_reference(gpu):
    g = golden("joint_gray_d3")
    im = g["image"].copy()
    gpu.JointBilateral.apply(im, g["image"].copy(), 8.0, 8.0, 0.0, 0.1)
    assert rel_err(im, g["joint"]) <= RTOL_FP32


def test_gauss_transform_reference_test_shape(gpu):
    g = golden("gt_reference_test")
    out = gpu.GaussTransform.apply(g["slice"], g["splat"], g["values"], list(g["sigmas"]))
    assert rel_err(out, g["out_distinct"]) <= RTOL_FP32
    out = gpu.GaussTransform.apply(None, g["splat"], g["values"], list(g["sigmas"]))
    assert rel_err(out, g["out_same"]) <= RTOL_FP32


def test_joint_bilateral_reference_test_shape_d6(gpu):
    g = golden("jb_reference_test")
    im = g["image"].copy()
    gpu.JointBilateral.apply(im, g["reference"], float(g["fw"]), float(g["fh"]), float(g["ft"]),
                             float(g["cs"]))
    assert rel_err(im, g["out"]) <= RTOL_FP32


def config1_points():
    rgb = synth.image(512, 512, 3, rects=16, seed=606)
    h, w = 512, 512
    p = np.empty((h, w, 5), np.float32)
    p[:, :, 0] = np.arange(w, dtype=np.float32)[None, :] * (np.float32(1) / np.float32(8))
    p[:, :, 1] = np.arange(h, dtype=np.float32)[:, None] * (np.float32(1) / np.float32(8))
    for k in range(3):
        p[:, :, 2 + k] = rgb[k] * (np.float32(1) / np.float32(0.1))
    v = np.concatenate([rgb.transpose(1, 2, 0), np.ones((h, w, 1), np.float32)], 2)
    return p.reshape(-1, 5), v.reshape(-1, 4).astype(np.float32)


def test_config1_512_bit_exact_keys_and_replay(gpu):
    g = golden("gt_config1_512")
    p, v = config1_points()
    d = gpu.lattice_dump(p, v)
    assert d["keys"].shape[0] == int(g["vertices"])
    assert sha(d["keys"]) == str(g["keys_sha256"])
    assert sha(d["replay_vtx"]) == str(g["replay_vtx_sha256"])
    assert sha(d["replay_w"]) == str(g["replay_w_sha256"])
    assert rel_err(d["out"][g["rows"]], g["out_rows"]) <= RTOL_FP32
    # a checksum of checksums: per-channel sums of the vertex values
    np.testing.assert_allclose(d["splat"].astype(np.float64).sum(0), g["sum_splat"], rtol=1e-5)
    np.testing.assert_allclose(d["blur"].astype(np.float64).sum(0), g["sum_blur"], rtol=1e-5)


def test_runs_are_deterministic_in_keys(gpu):
    p, v = config1_points()
    a = gpu.lattice_dump(p[:50000], v[:50000])
    b = gpu.lattice_dump(p[:50000], v[:50000])
    np.testing.assert_array_equal(a["keys"], b["keys"])
    np.testing.assert_array_equal(a["replay_vtx"], b["replay_vtx"])


def test_device_memory_path_matches_host(gpu):
    import torch
    img = synth.image(300, 200, 3, rects=10, seed=7)
    host = img.copy()
    gpu.Bilateral.apply(host, 6.0, 6.0, 0.0, 0.12)
    dev = torch.from_numpy(img.copy()).cuda()
    gpu.Bilateral.apply(dev, 6.0, 6.0, 0.0, 0.12)
    torch.cuda.synchronize()
    assert rel_err(dev.cpu().numpy(), host) <= RTOL_FP32


def test_strided_region_views(gpu):
    """A region of a larger image (the reference's Image views share the payload)."""
    big = synth.image(160, 120, 4, rects=6, seed=8)
    sub = big[:3, 10:90, 20:140]
    expect = np.ascontiguousarray(sub).copy()
    gpu.Bilateral.apply(expect, 5.0, 5.0, 0.0, 0.1)
    work = big.copy()
    gpu.Bilateral.apply(work[:3, 10:90, 20:140], 5.0, 5.0, 0.0, 0.1)
    assert rel_err(work[:3, 10:90, 20:140], expect) <= RTOL_FP32
    np.testing.assert_array_equal(work[3], big[3])            # untouched channel
    np.testing.assert_array_equal(work[:3, :10], big[:3, :10])  # untouched rows


@pytest.mark.parametrize("shape,fw,fh", [
    ((3, 1, 1), 4.0, 4.0),      # one pixel
    ((3, 1, 37), 4.0, 4.0),     # one row: the height axis drops out
    ((3, 29, 1), 4.0, 4.0),     # one column
    ((3, 12, 17), 0.0, 3.0),    # filter width 0: each column independently
    ((3, 12, 17), 3.0, 0.0),    # filter height 0: each row independently
    ((3, 20, 30), 500.0, 3.0),  # sigma > 10 x width: x is not a position
])
def test_degenerate_axes_match_reference_rules(gpu, shape, fw, fh):
    img = synth.image(shape[2], shape[1], shape[0], rects=2, seed=9)
    ours = img.copy()
    gpu.JointBilateral.apply(ours, img.copy(), fw, fh, 0.0, 0.2)
    if oracle.reference_available():
        ref, _ = oracle.reference_joint_bilateral(img, img, fw, 0.2, sigma_s_y=fh)
        assert rel_err(ours, ref) <= RTOL_FP32
    assert np.isfinite(ours).all()


def test_overfull_table_retry_keeps_input_intact(gpu):
    """A smooth frame teaches the engine a small vertex-per-pixel ratio; the next, noisy
    frame with the same d overflows the first table and is rerun with more slots.  The
    in-place output must equal a clean run's."""
    flat = np.full((3, 64, 64), 0.5, np.float32)
    gpu.Bilateral.apply(flat, 16.0, 16.0, 0.0, 0.5)
    rng = np.random.default_rng(5)
    noisy = rng.random((3, 64, 64), dtype=np.float32)
    out = noisy.copy()
    gpu.Bilateral.apply(out, 1.0, 1.0, 0.0, 0.02)
    assert gpu.last_stats()["retries"] >= 1
    pos, val = oracle.bilateral_points(noisy, noisy, 1.0, 0.02)
    ref = oracle.oracle_lattice(pos, val)
    norm = (ref.out[:, :3] / ref.out[:, 3:4]).reshape(64, 64, 3).transpose(2, 0, 1)
    assert rel_err(out, norm) <= RTOL_FP32


def test_errors_are_reported(gpu):
    img = np.zeros((3, 8, 8), np.float32)
    with pytest.raises(gpu.PgpuError) as e:
        gpu.JointBilateral.apply(img, np.zeros((3, 8, 9), np.float32), 2.0, 2.0, 0.0, 0.1)
    assert e.value.code == gpu.ERR_ARGUMENT
    with pytest.raises(gpu.PgpuError) as e:
        gpu.GaussTransform.apply(None, np.zeros((17, 1, 4, 4), np.float32),
                                 np.ones((2, 1, 4, 4), np.float32), [1.0] * 17)
    assert e.value.code == gpu.ERR_UNSUPPORTED
    with pytest.raises(gpu.PgpuError) as e:   # keys would leave the int16 range
        gpu.GaussTransform.apply(None, np.full((3, 1, 4, 4), 1e6, np.float32),
                                 np.ones((2, 1, 4, 4), np.float32), [1.0] * 3)
    assert e.value.code == gpu.ERR_ARGUMENT


def test_full_size_4k_bit_exact_vs_oracle(gpu, monkeypatch):
    """3840x2160 RGB, sigma_s 16, sigma_r 0.1: the whole vertex set and output, the output
    by both row layouts (slot-space rows with a compaction; vertex-ordered rows filled by
    the splat), each with either neighbour search."""
    img = synth.image(3840, 2160, 3, rects=64, seed=2)
    pos, val = oracle.bilateral_points(img, img, 16.0, 0.1)
    ref = oracle.oracle_lattice(pos, val)
    d = gpu.lattice_dump(pos, val)
    assert d["keys"].shape == ref.keys.shape
    assert sha(d["keys"]) == sha(ref.keys)
    assert sha(d["replay_vtx"]) == sha(ref.replay_vtx)
    assert sha(d["replay_w"]) == sha(ref.replay_w)
    assert rel_err(d["out"], ref.out) <= RTOL_FP32
    norm = (ref.out[:, :3] / ref.out[:, 3:4]).reshape(2160, 3840, 3).transpose(2, 0, 1)
    for rows, nbr in (("slot", "both"), ("slot", "half"), ("vertex", "both"), ("vertex", "half")):
        monkeypatch.setenv("PGPU_ROWS", rows)
        monkeypatch.setenv("PGPU_NBR", nbr)
        out = img.copy()
        gpu.Bilateral.apply(out, 16.0, 16.0, 0.0, 0.1)
        assert gpu.last_stats()["vertex_rows"] == (rows == "vertex")
        assert gpu.last_stats()["nbr_half"] == (nbr == "half")
        assert rel_err(out, norm) <= RTOL_FP32, (rows, nbr)


def test_fp64_payload_matches_fp64_oracle(gpu):
    g = golden("lattice_rgb_d5")
    d = gpu.lattice_dump(g["pos"], g["val"], payload="fp64")
    ref = oracle.oracle_lattice(g["pos"], g["val"], fp64=True)
    np.testing.assert_array_equal(d["keys"], ref.keys)
    # outputs are returned as float32
    assert rel_err(d["out"], ref.out) <= 1e-6


@pytest.mark.parametrize("rows", ["slot", "vertex"])
@pytest.mark.parametrize("payload,tol", [("fp16", 1e-3), ("bf16", 1e-2)])
def test_low_precision_payload_error_vs_fp64(gpu, monkeypatch, payload, tol, rows):
    """16-bit payloads against the FP64 lattice, with rows compacted from slot space or
    filled in vertex order by the splat (FP32 sums the first blur pass normalises)."""
    img = synth.image(512, 512, 3, rects=16, seed=11)
    ref = img.copy()
    gpu.Bilateral.apply(ref, 8.0, 8.0, 0.0, 0.1, payload="fp64")
    monkeypatch.setenv("PGPU_ROWS", rows)
    out = img.copy()
    gpu.Bilateral.apply(out, 8.0, 8.0, 0.0, 0.1, payload=payload)
    assert gpu.last_stats()["vertex_rows"] == (rows == "vertex")
    err = rel_err(out, ref, floor_frac=1e-2)
    print(payload, "max relative error vs FP64 lattice:", err)
    assert err <= tol


def test_exact_gauss_transform_f64_matches_oracle(gpu):
    """The GPU FP64 brute-force transform (the error oracle) against the C oracle's FP64
    brute force, and the lattice's own error against it (reported: the permutohedral
    lattice approximates the Gaussian, so only a loose bound holds)."""
    import torch
    g = golden("lattice_rgb_d5")
    pos, val = g["pos"], g["val"]
    rng = np.random.default_rng(5)
    qi = rng.choice(pos.shape[0], 64, replace=False)
    cpu = oracle.exact_gauss_transform(pos[qi], pos, val)
    dev = gpu.exact_gauss_transform_f64(torch.from_numpy(pos[qi]).cuda(),
                                        torch.from_numpy(pos).cuda(),
                                        torch.from_numpy(val).cuda()).cpu().numpy()
    assert rel_err(dev, cpu, floor_frac=1e-12) <= 1e-10
    lat = gpu.lattice_dump(pos, val)["out"][qi]
    norm = lambda a: a[:, :-1] / a[:, -1:]
    err = rel_err(norm(lat), norm(cpu), floor_frac=1e-2)
    print("lattice vs exact Gauss transform, max relative error:", err)
    assert err < 0.5


def test_red_probe_does_the_adds_it_times(gpu):
    """The atomic-roofline probe: two launches (warm-up, timed) of blocks x 256 threads,
    each adding a float4 of ones `per_thread` times at scattered rows."""
    import ctypes as C

    import torch
    rows, per_thread, blocks = 1 << 16, 8, 64
    table = torch.zeros((rows, 4), dtype=torch.float32, device="cuda")
    rate = C.c_double(0.0)
    rc = gpu.lib().pgpu_probe_red_rate(table.data_ptr(), rows, per_thread, blocks, None,
                                      C.byref(rate))
    assert rc == 0 and rate.value > 0
    assert float(table.sum().item()) == 2 * blocks * 256 * per_thread * 4


def test_nlmeans_filter_shape_d8_matches_reference(gpu):
    """NLMeans::apply's filter (src/GaussTransform.cpp:867-874): the image joint-bilateral
    filtered against patch features, frames INF, so d = 6 + 2 = 8 and keys of two words."""
    g = golden("nlmeans_d8")
    im = g["image"].copy()
    gpu.JointBilateral.apply(im, g["guide"], float(g["sigma_s"]), float(g["sigma_s"]),
                             float("inf"), float(g["sigma_p"]))
    assert gpu.last_stats()["d"] == 8
    assert rel_err(im, g["out"]) <= RTOL_FP32


def test_nlmeans3d_filter_shape_matches_reference(gpu):
    """NLMeans3D::apply's filter (src/GaussTransform.cpp:934-941): six frames against the
    reference's own 6-channel PCA guide, frames INF, so every frame's points go into one
    lattice of d = 8 without a t position; its vertex count is the reference's."""
    g = golden("nlmeans3d_d8")
    im = g["image"].copy()
    gpu.JointBilateral.apply(im, g["guide"], float(g["sigma_s"]), float(g["sigma_s"]),
                             float("inf"), float(g["sigma_p"]))
    st = gpu.last_stats()
    assert st["d"] == 8 and st["points"] == im[0].size
    assert st["vertices"] == int(g["vertices"])
    assert rel_err(im, g["out"]) <= RTOL_FP32


@pytest.mark.parametrize("key,sigma_t,d", [("t1_5", 1.5, 6), ("t0", 0.0, 5),
                                           ("tinf", float("inf"), 5)])
def test_video_frames_match_reference(gpu, key, sigma_t, d):
    """Bilateral::apply over five frames (src/GaussTransform.cpp:532-545): t as a
    position, each frame alone, and all frames in one lattice without a t position."""
    g = golden("video_frames")
    im = g["image"].copy()
    ss = float(g["sigma_s"])
    gpu.Bilateral.apply(im, ss, ss, sigma_t, float(g["sigma_r"]))
    st = gpu.last_stats()
    assert st["d"] == d
    if sigma_t != 0.0:   # one lattice over every frame
        assert st["points"] == im[0].size and st["vertices"] == int(g["vertices_" + key])
    assert rel_err(im, g["out_" + key]) <= RTOL_FP32


@pytest.mark.parametrize("method,key", [("permutohedral_gpu", "out_permutohedral"),
                                        ("grid_gpu", "out_grid")])
def test_chromablur_filter_shape_matches_reference(gpu, method, key):
    """ChromaBlur::apply's filter (src/GaussTransform.cpp:792-804): YUV against its
    luminance, by the lattice and by the grid (the method AUTO picks there).  U and V are
    signed and pass through zero, where summation order alone moves the last FP32 bits by
    more than 1e-5 of the value (the reference's own FP32 output is 1.4e-7 absolute from
    the FP64 lattice here), so the relative error is taken against max(|x|, 1e-3 max|x|)."""
    g = golden("chromablur_d3")
    im = g["image"].copy()
    gpu.JointBilateral.apply(im, g["guide"], float(g["sigma_s"]), float(g["sigma_s"]), 0.0,
                             float(g["sigma_c"]), method=method)
    err = rel_err(im, g[key], floor_frac=1e-3)
    print(method, "relative error against the reference:", err)
    assert err <= RTOL_FP32


def test_full_size_d16_gauss_transform_matches_reference_digests(gpu):
    """The 2,000,000-point d=16 Gauss transform (three key words, slot tags and the
    pending-slot protocol at full scale): the vertex count, the keys in vertex order and
    the replay records equal the reference's byte for byte, sampled outputs and
    per-channel value sums within 1e-5."""
    g = golden("gt_d16_2m")
    pos, val = synth.gauss_mixture(2_000_000, d=16, seed=2)
    d = gpu.lattice_dump(pos, val)
    assert d["keys"].shape[0] == int(g["vertices"])
    assert sha(d["keys"]) == str(g["keys_sha256"])
    assert sha(d["replay_vtx"]) == str(g["replay_vtx_sha256"])
    assert sha(d["replay_w"]) == str(g["replay_w_sha256"])
    # values are uniform in [-1, 1], so a channel's sum can cancel to near zero while the
    # splat's atomics (summing in another order than the reference) err relative to the
    # gross sum; the homogeneous weight in the last channel bounds that gross sum, so each
    # row's error is taken relative to its largest magnitude
    a = d["out"][g["rows"]].astype(np.float64)
    b = g["out_rows"].astype(np.float64)
    scale = np.abs(b).max(1, keepdims=True)
    assert float((np.abs(a - b) / scale).max()) <= RTOL_FP32
    np.testing.assert_allclose(d["splat"].astype(np.float64).sum(0), g["sum_splat"], rtol=1e-5, atol=1e-2)
    np.testing.assert_allclose(d["blur"].astype(np.float64).sum(0), g["sum_blur"], rtol=1e-5, atol=1e-2)


@pytest.mark.parametrize("mode", ["direct", "tile"])
def test_both_splat_kernels_bit_exact(gpu, monkeypatch, mode):
    """The direct splat (one point per thread, global table) and the tile splat (a
    shared-memory table per tile of points, then one global insert per distinct vertex)
    give the same keys, vertex order and replay records, bit for bit, and the same values
    within the FP32 tolerance (only their summation order differs)."""
    monkeypatch.setenv("PGPU_SPLAT", mode)
    g = golden("gt_config1_512")
    p, v = config1_points()
    d = gpu.lattice_dump(p, v)
    assert d["keys"].shape[0] == int(g["vertices"])
    assert sha(d["keys"]) == str(g["keys_sha256"])
    assert sha(d["replay_vtx"]) == str(g["replay_vtx_sha256"])
    assert sha(d["replay_w"]) == str(g["replay_w_sha256"])
    assert rel_err(d["out"][g["rows"]], g["out_rows"]) <= RTOL_FP32
    check_dump(gpu.lattice_dump(golden("lattice_rgb_d5")["pos"], golden("lattice_rgb_d5")["val"]),
               golden("lattice_rgb_d5"))


@pytest.mark.parametrize("mode", ["direct", "tile", "tile-vertex-rows"])
@pytest.mark.parametrize("w,h,c,ss,sr", [
    (333, 217, 3, 6.0, 0.1),    # tiles cut by both image edges
    (1000, 31, 1, 4.0, 0.2),    # fewer rows than a tile
    (17, 700, 3, 3.0, 0.15),    # narrower than a tile row
    (640, 480, 3, 2.0, 0.05),   # a sparse lattice: the tile tables overflow into the global one
])
def test_both_splat_kernels_match_the_oracle_on_images(gpu, monkeypatch, mode, w, h, c, ss, sr):
    """Bilateral filtering of images whose sizes do not divide into tiles, by each splat
    kernel, against the C oracle.  "tile-vertex-rows": the tile splat numbers the vertices
    as it creates them and accumulates into vertex-ordered rows (no compaction); the other
    modes keep rows in slot space with the compaction."""
    monkeypatch.setenv("PGPU_SPLAT", mode.split("-")[0])
    monkeypatch.setenv("PGPU_ROWS", "vertex" if mode == "tile-vertex-rows" else "slot")
    img = synth.image(w, h, c, rects=12, seed=w + h)
    out = img.copy()
    gpu.Bilateral.apply(out, ss, ss, 0.0, sr)
    pos, val = oracle.bilateral_points(img, img, ss, sr)
    ref = oracle.oracle_lattice(pos, val).out
    norm = (ref[:, :c] / ref[:, c:c + 1]).reshape(h, w, c).transpose(2, 0, 1)
    assert rel_err(out, norm) <= RTOL_FP32
