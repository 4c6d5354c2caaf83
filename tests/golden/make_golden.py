"""Generate the golden fixtures of tests/golden/ from the reference ImageStack itself.

Run in a checkout where the reference build exists (oracle/Makefile -> oracle/_ref):

    python tests/golden/make_golden.py

Every fixture is produced by the reference's own code (strict IEEE build), fed with the
seeded synthetic inputs of imagestack_b200.synth.  The reference's tests draw their inputs
from rand() seeded by the clock (src/main.cpp:67-75) and compare loosely
(src/main.cpp:45-48), so they pin nothing; these fixtures do.  Cases:

  lattice_rgb_d5        64x48 RGB bilateral positions (r,g,b,x,y), sigma_s 8, sigma_r 0.1:
                        the full lattice dump (keys, replay, splat, blur, slice)
  bilateral_rgb         Bilateral::apply of the same image
  gt_reference_test     the shape of GaussTransform::test (src/GaussTransform.cpp:39-77):
                        56x34x2 frames, 3 position channels, values (noise, 1),
                        sigma (0.2, 0.3, 0.4), distinct slice positions
  jb_reference_test     the shape of JointBilateral::test (src/GaussTransform.cpp:442-471):
                        60x50x3 frames, 3 channels, sigmas (3, 4, 1), colour 0.25 (d=6)
  joint_gray_d3         grey joint bilateral (lum, x, y), 96x64, sigma_s 8, sigma_r 0.1
  lattice_d16           d=16 Gaussian mixture, 1500 points, 4 values + 1 (the shape of
                        the high-dimensional Gauss transform workload)
  gt_config1_512        512x512 RGB, 16 rectangles, -gausstransform order (x/8, y/8,
                        r/0.1, g/0.1, b/0.1): SHA-256 digests of keys and replay records
                        and 4096 sampled output rows (the full arrays are tens of MB)
  nlmeans_d8            the shape of NLMeans::apply's filter (src/GaussTransform.cpp:867-874):
                        80x60 RGB joint-bilateral filtered against a 6-channel patch-feature
                        guide (linear mixes of shifted image channels, standing in for the
                        PCA projections), spatial sigma 4, patch sigma 0.3, frames INF, so
                        d = 6 + 2 = 8 (two key words)
  chromablur_d3         the shape of ChromaBlur::apply (src/GaussTransform.cpp:792-804): a
                        72x56 YUV image filtered against its luminance, sigmas (2, 0.5), by
                        the reference's PERMUTOHEDRAL and GRID methods (AUTO picks GRID for
                        three position channels)
  nlmeans3d_d8          the shape of NLMeans3D::apply (src/GaussTransform.cpp:934-941): a
                        40x32x6-frame RGB volume filtered against the reference's own PCA
                        guide (PatchPCA3D 5x5x5 patches -> 6 dimensions, Convolve), spatial
                        sigma 4, patch sigma 0.3, frames INF, so the six frames share one
                        lattice with d = 6 + 2 = 8 (the guide is stored: the reference
                        draws its patches at random)
  video_frames          Bilateral::apply of a 44x36x5-frame RGB volume (a moving image
                        plus noise), sigma_s 4, sigma_r 0.15, with sigma_t 1.5 (t is a
                        position, d = 6), 0 (each frame alone, d = 5) and INF (the frames
                        share one lattice without a t position, d = 5)
  gt_d16_2m             the full-size high-dimensional Gauss transform: 2,000,000 points of
                        synth.gauss_mixture(d=16, seed=2) (the benchmark's input), 4 values
                        + 1, unit sigmas, replay slice: vertex count, SHA-256 digests of the
                        keys and replay records, 4096 sampled output rows and per-channel
                        sums of the vertex values (about 5 minutes of reference CPU time;
                        `python tests/golden/make_golden.py gt_d16_2m` makes only this one)
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from imagestack_b200 import synth  # noqa: E402


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def save(name: str, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, os.path.getsize(path), "bytes")


def dump_arrays(prefix: str, d: oracle.LatticeDump) -> dict:
    return {prefix + "keys": d.keys, prefix + "replay_vtx": d.replay_vtx,
            prefix + "replay_w": d.replay_w, prefix + "splat": d.splat,
            prefix + "blur": d.blur, prefix + "out": d.out}


def main():
    if not oracle.reference_available():
        raise SystemExit("oracle/_ref is not built: run make -C oracle ref")

    # 1. lattice dump + Bilateral::apply, RGB d=5
    img = synth.image(64, 48, 3, rects=8, seed=101)
    pos, val = oracle.bilateral_points(img, img, 8.0, 0.1)
    dump = oracle.reference_lattice(pos, val)
    out, _ = oracle.reference_bilateral(img, 8.0, 0.1)
    save("lattice_rgb_d5", image=img, pos=pos, val=val, sigma_s=np.float32(8.0),
         sigma_r=np.float32(0.1), bilateral=out, **dump_arrays("", dump))

    # 2. GaussTransform::test shape: distinct slice positions (re-elevation slice)
    w, h, f = 56, 34, 2
    splat = synth.uniform(202, 1, 3 * f * h * w).astype(np.float32).reshape(3, f, h, w)
    slc = synth.uniform(202, 2, 3 * f * h * w).astype(np.float32).reshape(3, f, h, w)
    values = np.empty((2, f, h, w), np.float32)
    values[0] = synth.uniform(202, 3, f * h * w).astype(np.float32).reshape(f, h, w)
    values[1] = 1.0
    sig = np.array([0.2, 0.3, 0.4], np.float32)
    gt_out, _ = oracle.reference_gauss_transform(slc, splat, values, sig)
    gt_same, _ = oracle.reference_gauss_transform(None, splat, values, sig)
    save("gt_reference_test", splat=splat, slice=slc, values=values, sigmas=sig,
         out_distinct=gt_out, out_same=gt_same)

    # 3. JointBilateral::test shape (d = 3 colour + x + y + t = 6)
    w, h, f = 60, 50, 3
    im = synth.uniform(303, 1, 3 * f * h * w).astype(np.float32).reshape(3, f, h, w)
    ref = synth.uniform(303, 2, 3 * f * h * w).astype(np.float32).reshape(3, f, h, w)
    jb_out, _ = oracle.reference_joint_bilateral(im, ref, 3.0, 0.25, sigma_t=1.0, sigma_s_y=4.0)
    save("jb_reference_test", image=im, reference=ref, fw=np.float32(3), fh=np.float32(4),
         ft=np.float32(1), cs=np.float32(0.25), out=jb_out)

    # 4. grey joint bilateral, d = 3
    rgb = synth.image(96, 64, 3, rects=8, seed=404)
    lum = synth.luminance(rgb)
    gpos, gval = oracle.bilateral_points(lum, lum, 8.0, 0.1)
    gdump = oracle.reference_lattice(gpos, gval)
    gout, _ = oracle.reference_joint_bilateral(lum, lum, 8.0, 0.1)
    save("joint_gray_d3", image=lum, pos=gpos, val=gval, joint=gout, **dump_arrays("", gdump))

    # 5. d = 16 Gaussian mixture
    p16, v16 = synth.gauss_mixture(1500, d=16, seed=505)
    d16 = oracle.reference_lattice(p16, v16)
    save("lattice_d16", pos=p16, val=v16, **dump_arrays("", d16))

    # 6. config-1 shape, -gausstransform order: digests only
    rgb = synth.image(512, 512, 3, rects=16, seed=606)
    h, w = 512, 512
    p = np.empty((h, w, 5), np.float32)
    p[:, :, 0] = np.arange(w, dtype=np.float32)[None, :] * (np.float32(1) / np.float32(8))
    p[:, :, 1] = np.arange(h, dtype=np.float32)[:, None] * (np.float32(1) / np.float32(8))
    for k in range(3):
        p[:, :, 2 + k] = rgb[k] * (np.float32(1) / np.float32(0.1))
    v = np.concatenate([rgb.transpose(1, 2, 0), np.ones((h, w, 1), np.float32)], 2)
    p = p.reshape(-1, 5)
    v = v.reshape(-1, 4).astype(np.float32)
    big = oracle.reference_lattice(p, v)
    rows = (synth.uniform(607, 1, 4096) * (h * w)).astype(np.int64)
    save("gt_config1_512", vertices=np.int64(big.keys.shape[0]),
         keys_sha256=np.array(digest(big.keys)), replay_vtx_sha256=np.array(digest(big.replay_vtx)),
         replay_w_sha256=np.array(digest(big.replay_w)), rows=rows, out_rows=big.out[rows],
         sum_splat=big.splat.astype(np.float64).sum(0), sum_blur=big.blur.astype(np.float64).sum(0))


def gt_d16_2m():
    """The high-dimensional Gauss transform at its full size, pinned by digests."""
    pos, val = synth.gauss_mixture(2_000_000, d=16, seed=2)
    big = oracle.reference_lattice(pos, val)
    rows = (synth.uniform(1616, 1, 4096) * pos.shape[0]).astype(np.int64)
    save("gt_d16_2m", vertices=np.int64(big.keys.shape[0]),
         keys_sha256=np.array(digest(big.keys)), replay_vtx_sha256=np.array(digest(big.replay_vtx)),
         replay_w_sha256=np.array(digest(big.replay_w)), rows=rows, out_rows=big.out[rows],
         sum_splat=big.splat.astype(np.float64).sum(0), sum_blur=big.blur.astype(np.float64).sum(0))


def high_d_callers():
    """Fixtures of the reference's own callers of JointBilateral::apply beyond the bilateral
    filter: NLMeans (d = PCA dimensions + 2) and ChromaBlur (d = 3)."""
    rgb = synth.image(80, 60, 3, rects=10, seed=808)
    mix = (synth.uniform(808, 3, 6 * 3 * 5).astype(np.float32) * 2.0 - 1.0).reshape(6, 3, 5)
    shifts = [(0, 0), (0, 1), (1, 0), (0, -1), (-1, 0)]
    guide = np.zeros((6, 60, 80), np.float32)
    for k in range(6):
        for c in range(3):
            for j, (dy, dx) in enumerate(shifts):
                guide[k] += mix[k, c, j] * np.roll(rgb[c], (dy, dx), axis=(0, 1))
    inf = float("inf")
    nl_out, _ = oracle.reference_joint_bilateral(rgb, guide, 4.0, 0.3, sigma_t=inf)
    save("nlmeans_d8", image=rgb, guide=guide, sigma_s=np.float32(4), sigma_p=np.float32(0.3),
         out=nl_out)

    rgb = synth.image(72, 56, 3, rects=8, seed=909)
    y = 0.299 * rgb[0] + 0.587 * rgb[1] + 0.114 * rgb[2]
    yuv = np.stack([y, 0.492 * (rgb[2] - y), 0.877 * (rgb[0] - y)]).astype(np.float32)
    lum = y[None].astype(np.float32)
    perm, _ = oracle.reference_joint_bilateral(yuv, lum, 2.0, 0.5)
    grid, _ = oracle.reference_joint_bilateral(yuv, lum, 2.0, 0.5, method="grid")
    save("chromablur_d3", image=yuv, guide=lum, sigma_s=np.float32(2), sigma_c=np.float32(0.5),
         out_permutohedral=perm, out_grid=grid)



def volume_callers():
    """Fixtures over several frames: the three ways JointBilateral::apply treats the frame
    axis (a position, each frame alone, no position) and NLMeans3D's filter."""
    inf = float("inf")
    vol = np.stack([np.roll(synth.image(44, 36, 3, rects=6, seed=1100), 2 * t, axis=2) +
                    0.05 * synth.uniform(1200 + t, 1, 3 * 36 * 44).reshape(3, 36, 44)
                    for t in range(5)], 1).astype(np.float32)
    outs = {}
    for key, ft in (("t1_5", 1.5), ("t0", 0.0), ("tinf", inf)):
        outs["out_" + key], _ = oracle.reference_bilateral(vol, 4.0, 0.15, sigma_t=ft)
        if ft != 0.0:   # one lattice over every frame: its vertex count
            pos, val = oracle.volume_points(vol, vol, 4.0, 0.15, ft)
            outs["vertices_" + key] = np.int64(oracle.reference_lattice(pos, val).keys.shape[0])
    save("video_frames", image=vol, sigma_s=np.float32(4), sigma_r=np.float32(0.15), **outs)

    vol = np.stack([synth.image(40, 32, 3, rects=6, seed=1000 + t) for t in range(6)], 1)
    out, guide, _ = oracle.reference_nlmeans3d(vol, 0.5, 6, 4.0, 0.3)
    pos, val = oracle.volume_points(vol, guide, 4.0, 0.3, inf)
    save("nlmeans3d_d8", image=vol, guide=guide, patch=np.float32(0.5), dims=np.int32(6),
         sigma_s=np.float32(4), sigma_p=np.float32(0.3), out=out,
         vertices=np.int64(oracle.reference_lattice(pos, val).keys.shape[0]))


if __name__ == "__main__":
    if sys.argv[1:] == ["high_d"]:   # only the fixtures of the high-dimensional callers
        high_d_callers()
    elif sys.argv[1:] == ["volumes"]:   # only the fixtures over several frames
        volume_callers()
    elif sys.argv[1:] == ["gt_d16_2m"]:
        gt_d16_2m()
    else:
        main()
        high_d_callers()
        volume_callers()
        gt_d16_2m()
