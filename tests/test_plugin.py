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
