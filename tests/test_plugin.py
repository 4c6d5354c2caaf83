"""The drop-in path: the reference ImageStack CLI (oracle/_ref/ImageStack, built from the
reference sources) with `-plugin libpermgpu_imagestack.so`, images exchanged as .tmp files
(the reference's raw float format, src/FileTMP.cpp), read and written by
imagestack_b200.tmpfile."""
import os
import subprocess

import numpy as np
import pytest

import imagestack_b200 as ib
import oracle
from imagestack_b200 import synth
from imagestack_b200.tmpfile import load_tmp, save_tmp

PLUGIN = os.path.join(os.path.dirname(ib.LIB_PATH), "libpermgpu_imagestack.so")
needs_cli = pytest.mark.skipif(not (os.path.exists(oracle.REF_CLI) and os.path.exists(PLUGIN)),
                               reason="reference CLI or plugin not built")


def run_cli(args, tmp_path, plugin=True):
    cmd = [oracle.REF_CLI] + (["-plugin", PLUGIN] if plugin else []) + args
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=tmp_path, timeout=600)
    return r.stdout + r.stderr


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    floor = np.abs(b).max() * 1e-6
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max())


@needs_cli
def test_plugin_loads_and_extends_help(tmp_path):
    out = run_cli(["-help", "bilateral"], tmp_path)
    assert "permutohedral_gpu" in out


@needs_cli
def test_plugin_leaves_cpu_methods_unchanged(tmp_path):
    img = synth.image(40, 30, 3, rects=4, seed=3)
    save_tmp(tmp_path / "in.tmp", img)
    args = ["-load", "in.tmp", "-bilateral", "0.1", "4", "4", "0", "permutohedral", "-save", "out.tmp"]
    run_cli(args, tmp_path, plugin=False)
    a = load_tmp(tmp_path / "out.tmp")
    run_cli(args, tmp_path, plugin=True)
    b = load_tmp(tmp_path / "out.tmp")
    np.testing.assert_array_equal(a, b)


@needs_cli
@pytest.mark.skipif(ib.device_count() > 0, reason="checks the no-GPU behaviour")
def test_plugin_gpu_method_fails_loudly_without_gpu(tmp_path):
    img = synth.image(16, 16, 3, rects=2, seed=3)
    save_tmp(tmp_path / "in.tmp", img)
    out = run_cli(["-load", "in.tmp", "-bilateral", "0.1", "4", "4", "0", "permutohedral_gpu",
                   "-save", "out.tmp"], tmp_path)
    assert "permutohedral_gpu" in out and "device" in out
    assert not (tmp_path / "out.tmp").exists()


@needs_cli
@pytest.mark.gpu
def test_cli_bilateral_gpu_matches_cli_cpu(tmp_path):
    img = synth.image(320, 240, 3, rects=8, seed=4)
    save_tmp(tmp_path / "in.tmp", img)
    cpu = ["-load", "in.tmp", "-bilateral", "0.1", "8", "8", "0", "permutohedral", "-save", "cpu.tmp"]
    gpu = ["-load", "in.tmp", "-bilateral", "0.1", "8", "8", "0", "permutohedral_gpu", "-save", "gpu.tmp"]
    run_cli(cpu, tmp_path)
    log = run_cli(gpu, tmp_path)
    assert (tmp_path / "gpu.tmp").exists(), log
    assert rel_err(load_tmp(tmp_path / "gpu.tmp"), load_tmp(tmp_path / "cpu.tmp")) <= 1e-5


@needs_cli
@pytest.mark.gpu
def test_cli_jointbilateral_and_gausstransform_gpu_match_cpu(tmp_path):
    img = synth.image(200, 150, 3, rects=8, seed=5)
    ref = synth.luminance(synth.image(200, 150, 3, rects=8, seed=6))
    save_tmp(tmp_path / "im.tmp", img)
    save_tmp(tmp_path / "ref.tmp", ref)
    for m in ("permutohedral", "permutohedral_gpu"):
        run_cli(["-load", "ref.tmp", "-load", "im.tmp", "-jointbilateral", "0.1", "6", "6", "0", m,
                 "-save", "jb_%s.tmp" % m], tmp_path)
    assert rel_err(load_tmp(tmp_path / "jb_permutohedral_gpu.tmp"),
                   load_tmp(tmp_path / "jb_permutohedral.tmp")) <= 1e-5
    # -gausstransform with user-built positions (x, y, r, g, b) and values (r, g, b, 1):
    # the stack holds values, splat positions, slice positions (top)
    c, h, w = img.shape
    pos = np.empty((5, h, w), np.float32)
    pos[0] = np.arange(w, dtype=np.float32)[None, :]
    pos[1] = np.arange(h, dtype=np.float32)[:, None]
    pos[2:] = img
    vals = np.concatenate([img, np.ones((1, h, w), np.float32)], 0)
    save_tmp(tmp_path / "pos.tmp", pos)
    save_tmp(tmp_path / "vals.tmp", vals)
    for m in ("permutohedral", "permutohedral_gpu"):
        run_cli(["-load", "vals.tmp", "-load", "pos.tmp", "-dup", "-gausstransform", m,
                 "6", "6", "0.1", "0.1", "0.1", "-save", "gt_%s.tmp" % m], tmp_path)
    assert rel_err(load_tmp(tmp_path / "gt_permutohedral_gpu.tmp"),
                   load_tmp(tmp_path / "gt_permutohedral.tmp")) <= 1e-5


@needs_cli
@pytest.mark.gpu
def test_cli_operation_self_tests_pass_with_plugin(tmp_path):
    out = run_cli(["-test", "gausstransform", "jointbilateral", "bilateral"], tmp_path)
    assert out.count("Passed") >= 3 and "Failed" not in out, out[-2000:]


@needs_cli
@pytest.mark.gpu
def test_cli_grid_gpu_matches_cli_grid(tmp_path):
    """-bilateral ... grid_gpu against the reference CLI's own grid method (a grey image:
    three position channels, where JointBilateral's AUTO picks the grid)."""
    img = synth.luminance(synth.image(240, 160, 3, rects=8, seed=7))
    save_tmp(tmp_path / "in.tmp", img)
    for m in ("grid", "grid_gpu"):
        run_cli(["-load", "in.tmp", "-bilateral", "0.1", "8", "8", "0", m, "-save", "g_%s.tmp" % m],
                tmp_path)
    assert rel_err(load_tmp(tmp_path / "g_grid_gpu.tmp"), load_tmp(tmp_path / "g_grid.tmp")) <= 1e-5


# The operations that end in JointBilateral::apply (src/GaussTransform.cpp:739-941).
CALLERS = ("nlmeans", "nlmeans3d", "chromablur", "bilateralsharpen")


@needs_cli
def test_plugin_callers_help_and_cpu_paths_unchanged(tmp_path):
    """-chromablur and -bilateralsharpen without a method token are the reference's own
    operations (deterministic, so the outputs are compared bit for bit); every caller's
    help names the GPU method."""
    for name in CALLERS:
        assert "permutohedral_gpu" in run_cli(["-help", name], tmp_path)
    img = synth.image(48, 36, 3, rects=4, seed=3)
    save_tmp(tmp_path / "in.tmp", img)
    for op in (["-chromablur", "2", "0.5"], ["-bilateralsharpen", "4", "0.2", "0.5"]):
        args = ["-load", "in.tmp"] + op + ["-save", "out.tmp"]
        run_cli(args, tmp_path, plugin=False)
        a = load_tmp(tmp_path / "out.tmp")
        run_cli(args, tmp_path, plugin=True)
        np.testing.assert_array_equal(load_tmp(tmp_path / "out.tmp"), a)


@needs_cli
def test_plugin_nlmeans3d_refuses_volumes_shorter_than_a_patch(tmp_path):
    """The reference's 3D patch sampler has no valid patch centre in a one-frame image (it
    samples out of bounds); the GPU path refuses it before any device call."""
    save_tmp(tmp_path / "in.tmp", synth.image(48, 36, 3, rects=4, seed=3))
    out = run_cli(["-load", "in.tmp", "-nlmeans3d", "0.5", "6", "4", "0.4", "permutohedral_gpu",
                   "-save", "out.tmp"], tmp_path)
    assert "do not fit" in out
    assert not (tmp_path / "out.tmp").exists()


@needs_cli
@pytest.mark.gpu
def test_cli_chromablur_and_bilateralsharpen_gpu_match_cpu(tmp_path):
    """-chromablur ... grid_gpu against the reference's -chromablur (AUTO: the grid for its
    three position channels) and -bilateralsharpen ... permutohedral_gpu against the
    reference's (AUTO: the lattice, d = 5).  Both outputs pass through zero (the colour
    round trip and the sharpening mix im * 1.5 - filtered * 0.5 leave pixels near 0), where
    summation order alone moves the last FP32 bits by more than 1e-5 of the value, so the
    error is taken against each output's largest magnitude."""
    img = synth.image(160, 120, 3, rects=8, seed=8)
    save_tmp(tmp_path / "in.tmp", img)
    run_cli(["-load", "in.tmp", "-chromablur", "2", "0.5", "-save", "cb_cpu.tmp"], tmp_path)
    log = run_cli(["-load", "in.tmp", "-chromablur", "2", "0.5", "grid_gpu", "-save", "cb_gpu.tmp"],
                  tmp_path)
    assert (tmp_path / "cb_gpu.tmp").exists(), log
    a, b = load_tmp(tmp_path / "cb_gpu.tmp"), load_tmp(tmp_path / "cb_cpu.tmp")
    assert float(np.abs(a - b).max()) <= 1e-5 * float(np.abs(b).max())
    run_cli(["-load", "in.tmp", "-bilateralsharpen", "8", "0.2", "0.5", "-save", "bs_cpu.tmp"],
            tmp_path)
    log = run_cli(["-load", "in.tmp", "-bilateralsharpen", "8", "0.2", "0.5", "permutohedral_gpu",
                   "-save", "bs_gpu.tmp"], tmp_path)
    assert (tmp_path / "bs_gpu.tmp").exists(), log
    a, b = load_tmp(tmp_path / "bs_gpu.tmp"), load_tmp(tmp_path / "bs_cpu.tmp")
    assert float(np.abs(a - b).max()) <= 1e-5 * float(np.abs(b).max())


@needs_cli
@pytest.mark.gpu
@pytest.mark.parametrize("op,patch,frames", [("-nlmeans", "1", 1), ("-nlmeans3d", "0.5", 6)])
def test_cli_nlmeans_gpu_denoises_like_cpu(tmp_path, op, patch, frames):
    """-nlmeans / -nlmeans3d with the GPU filter.  The reference draws its PCA patches at
    random (rand() seeded by the clock), so two runs filter against different guides: the
    GPU run must remove as much noise as the reference's own run (uniform noise of +-0.2;
    the reference leaves 0.039-0.042 mean absolute error of the 0.10 it was given)."""
    if frames == 1:
        clean = synth.image(96, 72, 3, rects=6, seed=41)
    else:
        clean = np.stack([synth.image(40, 32, 3, rects=4, seed=50)] * frames, 1)
    noise = (synth.uniform(42, 1, clean.size).reshape(clean.shape) * 0.4 - 0.2).astype(np.float32)
    save_tmp(tmp_path / "noisy.tmp", clean + noise)
    args = [patch, "6", "8", "0.3"]
    run_cli(["-load", "noisy.tmp", op] + args + ["permutohedral", "-save", "cpu.tmp"], tmp_path)
    log = run_cli(["-load", "noisy.tmp", op] + args + ["permutohedral_gpu", "-save", "gpu.tmp"],
                  tmp_path)
    assert (tmp_path / "gpu.tmp").exists(), log
    err_cpu = float(np.abs(load_tmp(tmp_path / "cpu.tmp") - clean).mean())
    err_gpu = float(np.abs(load_tmp(tmp_path / "gpu.tmp") - clean).mean())
    print(op, "mean abs error: noisy", float(np.abs(noise).mean()), "cpu", err_cpu, "gpu", err_gpu)
    assert err_gpu <= 0.5 * float(np.abs(noise).mean())
    assert err_gpu <= 1.1 * err_cpu


@needs_cli
@pytest.mark.gpu
def test_cli_caller_self_tests_pass_with_plugin(tmp_path):
    """-test on the callers runs the plugin's checks: the GPU filter against the reference's
    on one PCA guide (NLMeans, NLMeans3D), -chromablur against the reference's grid and
    -bilateralsharpen against its lattice."""
    out = run_cli(["-test"] + list(CALLERS), tmp_path)
    assert out.count("Passed") >= 4 and "Failed" not in out, out[-2000:]
