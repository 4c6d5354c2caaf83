"""Batched bilateral filtering: many uneven images per launch, each with its own lattice
(its own hash-table range) and sigmas; every result must equal the single-image path."""
import numpy as np
import pytest

import imagestack_b200 as ib
from imagestack_b200 import synth

RTOL_FP32 = 1e-5


def rel_err(a, b, floor_frac=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    floor = max(np.abs(b).max() * floor_frac, 1e-30)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max())


def uneven_batch(count, seed, lo=64, hi=320, channels=3):
    specs = synth.batch_specs(count, lo, hi, seed=seed)
    imgs = [synth.image(w, h, channels, rects=6, seed=s) for (w, h, ss, sr, s) in specs]
    return imgs, [s[2] for s in specs], [s[3] for s in specs]


def test_batch_argument_checks_need_no_gpu():
    a = np.zeros((3, 20, 20), np.float32)
    b = np.zeros((1, 20, 20), np.float32)
    with pytest.raises(ib.PgpuError) as e:     # channel counts differ
        ib.bilateral_batch([a, b], [4.0, 4.0], [0.1, 0.1])
    assert e.value.code == ib.ERR_ARGUMENT
    with pytest.raises(ib.PgpuError) as e:     # sigma too large for a 20 px side
        ib.bilateral_batch([a], [400.0], [0.1])
    assert e.value.code == ib.ERR_UNSUPPORTED
    with pytest.raises(ib.PgpuError):
        ib.bilateral_batch([a], [4.0, 5.0], [0.1])


def test_queued_batch_argument_checks_need_no_gpu():
    """pgpu_bilateral_batch_submit refuses bad arguments before it touches a device: output
    views of another size, device memory, no images."""
    import ctypes as C
    a = np.zeros((3, 20, 24), np.float32)
    with pytest.raises(ib.PgpuError) as e:      # an output of another size
        ib.bilateral_batch_submit([a], [4.0], [0.1], outputs=[np.zeros((3, 20, 20), np.float32)])
    assert e.value.code == ib.ERR_ARGUMENT
    with pytest.raises(ib.PgpuError) as e:      # one output per image
        ib.bilateral_batch_submit([a, a.copy()], [4.0, 4.0], [0.1, 0.1], outputs=[a.copy()])
    assert e.value.code == ib.ERR_ARGUMENT
    with pytest.raises(ib.PgpuError) as e:      # no images
        ib.bilateral_batch_submit([], [], [])
    assert e.value.code == ib.ERR_ARGUMENT
    v, _ = ib._view(a, "image")
    opt = ib._options(ib.MEM_DEVICE, "fp32")
    fw, cs, t = (C.c_float * 1)(4.0), (C.c_float * 1)(0.1), C.c_longlong(0)
    rc = ib.lib().pgpu_bilateral_batch_submit(C.byref(v), None, 1, fw, cs, C.byref(opt), C.byref(t))
    assert rc == ib.ERR_ARGUMENT                # queued batches take host memory
    assert ib.lib().pgpu_batch_wait(0) == ib.ERR_ARGUMENT


def test_batched_views_equal_per_image_views():
    """The batched view builder writes the same pgpu_image fields as _view, for (c, h, w)
    and (c, f, h, w) tensors, cropped and channel-sliced ones included, and declines
    (returns None) whatever _view would reject."""
    torch = pytest.importorskip("torch")
    g = torch.Generator().manual_seed(0)
    ims = []
    for i in range(40):
        h, w = 16 + (i * 7) % 23, 16 + (i * 11) % 29
        t = torch.rand(3, h, w, generator=g)
        if i % 5 == 1:
            t = t[:, 1:, 2:]
        if i % 7 == 2:
            t = torch.rand(3, 2, h, w, generator=g)
        if i % 11 == 3:
            t = torch.rand(5, h, w + 3, generator=g)[1:4, :, :w]
        ims.append(t)
    views, mem = ib._views_torch(ims)
    assert mem == ib.MEM_HOST
    for i, t in enumerate(ims):
        v, m = ib._view(t, "image")
        assert m == mem
        for f, _ in ib.Image._fields_:
            assert getattr(views[i], f) == getattr(v, f), (i, f)
    assert ib._views_torch([torch.zeros(3, 4, 4, dtype=torch.float64)]) is None
    assert ib._views_torch([torch.zeros(3, 4, 4).transpose(1, 2)]) is None
    assert ib._views_torch([torch.zeros(4, 4)]) is None


@pytest.mark.gpu
def test_batch_matches_single_image_path(gpu):
    imgs, ss, sr = uneven_batch(24, seed=3)
    expect = []
    for im, s, r in zip(imgs, ss, sr):
        e = im.copy()
        gpu.Bilateral.apply(e, s, s, 0.0, r)
        expect.append(e)
    work = [im.copy() for im in imgs]
    gpu.bilateral_batch(work, ss, sr)
    st = gpu.last_stats()
    assert st["points"] == sum(im.shape[1] * im.shape[2] for im in imgs)
    for w, e in zip(work, expect):
        assert rel_err(w, e) <= RTOL_FP32


@pytest.mark.gpu
@pytest.mark.parametrize("pinned", [False, True])
def test_host_batch_in_overlapped_chunks(gpu, pinned):
    """A host batch of more than two chunks' pixels (chunks of 2^22 pixels) is uploaded,
    filtered and downloaded chunk by chunk on overlapping streams; every image must still
    equal the single-image path, and the statistics must cover the whole batch."""
    import torch
    # three chunks: images 0-2, 3-5, 6 (slot 0 is reused by the third)
    sizes = [(1920, 1200), (1600, 1000), (2048, 1152), (640, 480), (1280, 720), (2560, 1440),
             (1024, 1024)]
    imgs = [synth.image(w, h, 3, rects=12, seed=40 + k) for k, (w, h) in enumerate(sizes)]
    ss = [8.0, 12.0, 16.0, 6.0, 10.0, 14.0, 9.0]
    sr = [0.1, 0.15, 0.08, 0.2, 0.12, 0.1, 0.3]
    expect = []
    for im, s, r in zip(imgs, ss, sr):
        e = im.copy()
        gpu.Bilateral.apply(e, s, s, 0.0, r)
        expect.append(e)
    for rep in range(2):
        if pinned:
            keep = [torch.from_numpy(im.copy()).pin_memory() for im in imgs]
            work = [t.numpy() for t in keep]
        else:
            work = [im.copy() for im in imgs]
        gpu.bilateral_batch(work, ss, sr)
        st = gpu.last_stats()
        assert st["points"] == sum(w * h for w, h in sizes)
        for w, e in zip(work, expect):
            assert rel_err(w, e) <= RTOL_FP32


@pytest.mark.gpu
def test_batch_on_device_with_graph_replay(gpu):
    import torch
    imgs, ss, sr = uneven_batch(16, seed=4)
    expect = [im.copy() for im in imgs]
    gpu.bilateral_batch(expect, ss, sr)
    for rep in range(3):   # capture once, replay twice
        dev = [torch.from_numpy(im.copy()).cuda() for im in imgs]
        gpu.bilateral_batch(dev, ss, sr, graph=True)
        torch.cuda.synchronize()
        for d, e in zip(dev, expect):
            assert rel_err(d.cpu().numpy(), e) <= RTOL_FP32


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_autotuned_batch_tries_candidates_then_keeps_one(gpu, graph):
    """With autotune the first calls of a batch shape walk the knobs one at a time, each
    option timed twice: load factor 0.5 / 0.35 / 0.7, then one blur axis per pass, then one
    vertex per blur thread, then the direct splat; later calls keep the fastest setting.
    Every call's results equal the single-image path."""
    import torch
    imgs, ss, sr = uneven_batch(10 + int(graph), seed=12)
    expect = []
    for im, s, r in zip(imgs, ss, sr):
        e = im.copy()
        gpu.Bilateral.apply(e, s, s, 0.0, r)
        expect.append(e)
    seen = []
    for call in range(22):
        dev = [torch.from_numpy(im.copy()).cuda() for im in imgs]
        gpu.bilateral_batch(dev, ss, sr, graph=graph, autotune=True)
        st = gpu.last_stats()
        seen.append((round(st["load_factor"], 2), st["blur_pairs"], st["blur_grid"], st["tiled"] > 0,
                     st["tuned"], st["nbr_half"]))
        torch.cuda.synchronize()
        for d, e in zip(dev, expect):
            assert rel_err(d.cpu().numpy(), e) <= RTOL_FP32
    trials = [x for x in seen if x[4] == 1]
    n = len(trials)
    # 6 load trials, 2 direct splat, 2 vertex-ordered rows, 2 one-lookup neighbour searches
    # when vertex-ordered rows won, 2 one-axis blur, 2 or 4 blur grid (a third option when
    # one-axis passes won), 2 wider tiles
    assert 16 <= n <= 20 and all(x[4] == 1 for x in seen[:n])
    assert [x[0] for x in trials[:6]] == [0.5, 0.5, 0.35, 0.35, 0.7, 0.7]
    assert all(x[1:4] == (1, 0, True) for x in trials[:6])
    best_load = trials[6][0]
    assert best_load in (0.5, 0.35, 0.7) and all(x[0] == best_load for x in trials[6:])
    assert all(x[3] is False for x in trials[6:8])              # the direct splat, twice
    assert sum(1 for x in trials if x[1] == 0) >= 2             # one blur axis per pass
    assert sum(1 for x in trials if x[2] == 1) >= 2             # one vertex per blur thread
    assert seen[n] == seen[n + 1] and seen[n][4] == 2
    assert seen[n][:4] in [x[:4] for x in trials]


@pytest.mark.gpu
def test_autotuned_fp16_batch_stays_within_its_error_bound(gpu):
    """A 16-bit payload walks the same knobs (one axis per pass included: it rounds rows
    to 16 bits where fused pairs do) and stays within its error bound on every call."""
    imgs, ss, sr = uneven_batch(9, seed=13, lo=128, hi=384)
    ref = [im.copy() for im in imgs]
    gpu.bilateral_batch(ref, ss, sr, payload="fp64")
    seen = []
    for call in range(22):
        out = [im.copy() for im in imgs]
        gpu.bilateral_batch(out, ss, sr, payload="fp16", autotune=True)
        st = gpu.last_stats()
        seen.append((round(st["load_factor"], 2), st["blur_pairs"], st["tuned"]))
        assert max(rel_err(o, r, floor_frac=1e-2) for o, r in zip(out, ref)) <= 1e-3
    assert [l for l, _, _ in seen[:6]] == [0.5, 0.5, 0.35, 0.35, 0.7, 0.7]
    assert sum(1 for _, p, t in seen if p == 0 and t == 1) >= 2   # one axis per pass tried
    n = sum(1 for _, _, t in seen if t == 1)
    assert 16 <= n <= 20 and [t for _, _, t in seen] == [1] * n + [2] * (22 - n)


@pytest.mark.gpu
@pytest.mark.parametrize("payload,tol", [("fp16", 1e-3), ("bf16", 1e-2)])
@pytest.mark.parametrize("rows", ["slot", "vertex"])
def test_16bit_one_axis_passes_round_where_pairs_do(gpu, monkeypatch, payload, tol, rows):
    """16-bit rows blurred one axis per pass are kept in FP32 after the first axis of each
    would-be pair and rounded after the second, where a fused pair rounds them, so both
    forms compute the same arithmetic; the splat's atomic sums differ in order from run to
    run, so the two are compared through their error against the FP64 lattice (d = 5 and
    d = 3, both row layouts)."""
    import torch
    monkeypatch.setenv("PGPU_ROWS", rows)
    for c in (3, 1):
        imgs, ss, sr = uneven_batch(6, seed=50 + c, lo=128, hi=512, channels=c)
        ref = [torch.from_numpy(im.copy()).cuda() for im in imgs]
        monkeypatch.delenv("PGPU_BLUR", raising=False)
        gpu.bilateral_batch(ref, ss, sr, payload="fp64")
        torch.cuda.synchronize()
        ref = [r.cpu().numpy() for r in ref]
        for mode in ("pairs", "single"):
            monkeypatch.setenv("PGPU_BLUR", mode)
            dev = [torch.from_numpy(im.copy()).cuda() for im in imgs]
            gpu.bilateral_batch(dev, ss, sr, payload=payload)
            st = gpu.last_stats()
            assert st["blur_pairs"] == (mode == "pairs")
            assert rows == "vertex" or st["vertex_rows"] == 0
            torch.cuda.synchronize()
            err = max(rel_err(d.cpu().numpy(), r, floor_frac=1e-2) for d, r in zip(dev, ref))
            assert err <= tol, (mode, c, err)


def _expect_single(gpu, imgs, ss, sr):
    out = []
    for im, s, r in zip(imgs, ss, sr):
        e = im.copy()
        gpu.Bilateral.apply(e, s, s, 0.0, r)
        out.append(e)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("rows", ["slot", "vertex"])
def test_queued_batches_overlap_and_match_the_single_image_path(gpu, monkeypatch, rows):
    """Three queued host batches (out of place, pinned), in flight together and waited for
    out of order: every output equals the single-image path and no input is touched.  A
    batch of more than three chunks makes the device slots turn over within one batch and
    across batches.  Both row layouts."""
    import torch
    sizes = [(2304, 1830), (2048, 2048), (2560, 1640), (1920, 1080), (1200, 900)]
    imgs = [synth.image(w, h, 3, rects=12, seed=90 + k) for k, (w, h) in enumerate(sizes)]
    ss = [12.0, 16.0, 8.0, 10.0, 6.0]
    sr = [0.1, 0.12, 0.08, 0.15, 0.2]
    expect = _expect_single(gpu, imgs, ss, sr)
    monkeypatch.setenv("PGPU_ROWS", rows)
    keep_in = [torch.from_numpy(im.copy()).pin_memory() for im in imgs]
    keep_out = [[torch.empty(im.shape, dtype=torch.float32).pin_memory() for im in imgs]
                for _ in range(3)]
    ins = [t.numpy() for t in keep_in]
    outs = [[t.numpy() for t in row] for row in keep_out]
    tickets = [gpu.bilateral_batch_submit(ins, ss, sr, outputs=outs[k]) for k in range(3)]
    for k in (1, 0, 2):
        res = tickets[k].wait()
        for w, e in zip(res, expect):
            assert rel_err(w, e) <= RTOL_FP32
    for a, b in zip(ins, imgs):
        assert np.array_equal(a, b)
    st = gpu.last_stats()
    assert st["points"] == sum(w * h for w, h in sizes)


@pytest.mark.gpu
def test_queued_batch_in_place_then_other_calls_finish_it(gpu):
    """An in-place queued batch, then a synchronous call on the same device before its wait:
    the call finishes the queued batch first, and the wait then reports its outcome."""
    import torch
    imgs, ss, sr = uneven_batch(12, seed=31, lo=200, hi=900)
    expect = _expect_single(gpu, imgs, ss, sr)
    keep = [torch.from_numpy(im.copy()).pin_memory() for im in imgs]
    work = [k.numpy() for k in keep]
    t = gpu.bilateral_batch_submit(work, ss, sr)
    other = imgs[0].copy()
    gpu.Bilateral.apply(other, ss[0], ss[0], 0.0, sr[0])
    assert rel_err(other, expect[0]) <= RTOL_FP32
    t.wait()
    for w, e in zip(work, expect):
        assert rel_err(w, e) <= RTOL_FP32
    with pytest.raises(gpu.PgpuError) as e:      # a ticket is waited for once
        gpu._check(gpu.lib().pgpu_batch_wait(t.ticket))
    assert e.value.code == gpu.ERR_ARGUMENT


@pytest.mark.gpu
def test_queued_batch_reruns_an_overflowed_image_at_its_wait(gpu):
    """A flat image teaches a small vertex ratio; a queued batch then holds a noisy image of
    a new shape, sized from that ratio, which overflows: its output is filtered again when
    the batch is waited for, and every output equals the single-image path."""
    flat = np.full((3, 300, 280), 0.25, np.float32)
    gpu.bilateral_batch([flat.copy()], [16.0], [0.5])
    rng = np.random.default_rng(19)
    noisy = rng.random((3, 222, 333), dtype=np.float32)
    imgs = [flat, noisy]
    ss, sr = [16.0, 1.0], [0.5, 0.02]
    outs = [np.zeros_like(flat), np.zeros_like(noisy)]
    res = gpu.bilateral_batch_submit(imgs, ss, sr, outputs=outs).wait()
    assert gpu.last_stats()["retries"] >= 1
    expect = _expect_single(gpu, imgs, ss, sr)
    for w, e in zip(res, expect):
        assert rel_err(w, e) <= RTOL_FP32


@pytest.mark.gpu
def test_queued_batch_while_the_autotuner_times_runs_at_once(gpu):
    """A shape the autotuner is still timing is filtered before the submission returns;
    once it is tuned, later submissions are queued; all outputs are exact."""
    imgs, ss, sr = uneven_batch(6, seed=44, lo=128, hi=512)
    expect = _expect_single(gpu, imgs, ss, sr)
    for call in range(23):
        outs = [np.zeros_like(im) for im in imgs]
        t = gpu.bilateral_batch_submit(imgs, ss, sr, outputs=outs, autotune=True)
        if call < 16:   # every trial ran inside the submission (at least 16 trials)
            for w, e in zip(outs, expect):
                assert rel_err(w, e) <= RTOL_FP32
        for w, e in zip(t.wait(), expect):
            assert rel_err(w, e) <= RTOL_FP32


@pytest.mark.gpu
@pytest.mark.parametrize("payload,tol", [("fp32", RTOL_FP32), ("fp16", 1e-3)])
def test_vertex_rows_batch_with_direct_splat_images_runs_as_two(gpu, monkeypatch, payload, tol):
    """Vertex-ordered rows need every image of the launches on the tile splat: a batch
    that asks for them, with a sparse image the direct splat takes once its density is
    learned, runs as two (the tile-splat images with vertex-ordered rows); every output
    stays within its payload's tolerance of the FP64 lattice."""
    rng = np.random.default_rng(5)
    imgs = [synth.image(300 + 40 * k, 220 + 30 * k, 3, rects=8, seed=80 + k) for k in range(3)]
    imgs.append(rng.random((3, 96, 104), dtype=np.float32))         # sparse: direct splat
    ss, sr = [8.0, 10.0, 12.0, 1.0], [0.1, 0.12, 0.15, 0.02]
    monkeypatch.setenv("PGPU_ROWS", "slot")
    ref = [im.copy() for im in imgs]
    gpu.bilateral_batch(ref, ss, sr, payload="fp64")
    monkeypatch.setenv("PGPU_ROWS", "vertex")
    for call in range(2):   # the first call learns the sparse image's density
        work = [im.copy() for im in imgs]
        gpu.bilateral_batch(work, ss, sr, payload=payload)
        st = gpu.last_stats()
        for w, r in zip(work, ref):
            assert rel_err(w, r, floor_frac=1e-2) <= tol
    assert st["tiled"] == 3 and st["vertex_rows"] == 1
    assert st["points"] == sum(im.shape[1] * im.shape[2] for im in imgs)


@pytest.mark.gpu
def test_batch_fp16_payload_error_vs_fp64(gpu):
    imgs, ss, sr = uneven_batch(12, seed=5, lo=128, hi=512)
    ref = [im.copy() for im in imgs]
    gpu.bilateral_batch(ref, ss, sr, payload="fp64")
    out = [im.copy() for im in imgs]
    gpu.bilateral_batch(out, ss, sr, payload="fp16")
    err = max(rel_err(o, r, floor_frac=1e-2) for o, r in zip(out, ref))
    print("batched fp16 max relative error vs FP64 lattice:", err)
    assert err <= 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("on_device", [False, True])
def test_batch_retry_leaves_finished_images_alone(gpu, on_device):
    """A textured image learns its vertex ratio; in the next batch a noisy image with no
    learned ratio overflows its range and is rerun.  The textured image, finished in the
    first pass (in place), must not be filtered a second time."""
    import torch
    tex = synth.image(200, 150, 3, rects=8, seed=21)
    gpu.bilateral_batch([tex.copy()], [8.0], [0.1])
    rng = np.random.default_rng(22)
    # a shape of its own per variant: ratios are learned by shape and sigmas
    noisy = rng.random((3, 90, 70 + 7 * int(on_device)), dtype=np.float32)
    if on_device:
        work = [torch.from_numpy(tex.copy()).cuda(), torch.from_numpy(noisy.copy()).cuda()]
    else:
        work = [tex.copy(), noisy.copy()]
    gpu.bilateral_batch(work, [8.0, 1.0], [0.1, 0.02])
    assert gpu.last_stats()["retries"] >= 1
    if on_device:
        torch.cuda.synchronize()
        work = [w.cpu().numpy() for w in work]
    e0, e1 = tex.copy(), noisy.copy()
    gpu.Bilateral.apply(e0, 8.0, 8.0, 0.0, 0.1)
    gpu.Bilateral.apply(e1, 1.0, 1.0, 0.0, 0.02)
    assert rel_err(work[0], e0) <= RTOL_FP32
    assert rel_err(work[1], e1) <= RTOL_FP32


@pytest.mark.gpu
@pytest.mark.parametrize("rows", ["slot", "vertex"])
def test_batch_retries_only_what_overflows(gpu, monkeypatch, rows):
    """A flat image teaches a small vertex ratio; a noisy one in the same batch then
    overflows its range and is rerun; both results stay exact, with rows in slot space or
    numbered by the splat (whose waits for other blocks' vertex numbers must end when the
    table overflows)."""
    flat = np.full((3, 96, 96), 0.25, np.float32)
    gpu.bilateral_batch([flat.copy()], [16.0], [0.5])
    rng = np.random.default_rng(9)
    # a shape of its own per variant: ratios are learned by shape and sigmas
    noisy = rng.random((3, 80, 80 + 3 * (rows == "vertex")), dtype=np.float32)
    work = [flat.copy(), noisy.copy()]
    monkeypatch.setenv("PGPU_ROWS", rows)
    gpu.bilateral_batch(work, [16.0, 1.0], [0.5, 0.02])
    st = gpu.last_stats()
    assert st["retries"] >= 1 and st["vertex_rows"] == (rows == "vertex")
    monkeypatch.setenv("PGPU_ROWS", "slot")
    e0, e1 = flat.copy(), noisy.copy()
    gpu.Bilateral.apply(e0, 16.0, 16.0, 0.0, 0.5)
    gpu.Bilateral.apply(e1, 1.0, 1.0, 0.0, 0.02)
    assert rel_err(work[0], e0) <= RTOL_FP32
    assert rel_err(work[1], e1) <= RTOL_FP32


def _oracle_bilateral(img, ss, sr):
    """The C oracle's bilateral of one planar image (positions (c/sr, x/ss, y/ss), values
    (c, 1), normalised by the homogeneous channel)."""
    import oracle
    c, h, w = img.shape
    pos, val = oracle.bilateral_points(img, img, ss, sr)
    out = oracle.oracle_lattice(pos, val).out
    return (out[:, :c] / out[:, c:c + 1]).reshape(h, w, c).transpose(2, 0, 1)


@pytest.mark.gpu
def test_full_mixed_batch_matches_the_oracle_and_fp16_the_fp64_lattice(gpu):
    """The 256-image mixed batch at its real size (sides 128..1024, per-image sigmas), in
    one batched call from device memory.  FP32: the eight largest and eight smallest images
    equal the C oracle within 1e-5 — the oracle is pinned bit for bit to the reference, so
    this checks the batch's segment offsets where the images are large.  FP16 payload:
    every image within 1e-3 of the FP64 lattice (relative to max(|x|, 1e-2 max|x|))."""
    import torch
    specs = synth.batch_specs(256, 128, 1024, seed=2)
    imgs = [synth.image(w, h, 3, rects=16, seed=s) for (w, h, _, _, s) in specs]
    ss = [s[2] for s in specs]
    sr = [s[3] for s in specs]
    dev = [torch.from_numpy(im).cuda() for im in imgs]
    work = [d.clone() for d in dev]
    gpu.bilateral_batch(work, ss, sr, payload="fp32", graph=True)
    torch.cuda.synchronize()
    px = [im.shape[1] * im.shape[2] for im in imgs]
    order = np.argsort(px)
    for k in list(order[:8]) + list(order[-8:]):
        expect = _oracle_bilateral(imgs[k], ss[k], sr[k])
        assert rel_err(work[k].cpu().numpy(), expect) <= RTOL_FP32, "image %d (%d px)" % (k, px[k])
    half = [d.clone() for d in dev]
    gpu.bilateral_batch(half, ss, sr, payload="fp16", graph=True)
    torch.cuda.synchronize()
    for k in range(256):
        ref = dev[k].clone()
        gpu.Bilateral.apply(ref, ss[k], ss[k], 0.0, sr[k], payload="fp64")
        torch.cuda.synchronize()
        assert rel_err(half[k].cpu().numpy(), ref.cpu().numpy(), floor_frac=1e-2) <= 1e-3, k


@pytest.mark.gpu
def test_host_batch_of_large_images_one_per_chunk_with_an_overflow_rerun(gpu):
    """Images of at least 2^22 pixels are chunks of their own, each uploaded, filtered and
    downloaded on the overlapping streams.  Every image equals the single-image path,
    including a noisy one whose first table overflows (its shape is new, so its table size
    is guessed) and is rerun in the middle of the pipeline.  Odd heights on purpose."""
    import torch
    rng = np.random.default_rng(77)
    sizes = [(2304, 1830), (2111, 2003), (2560, 1640)]
    imgs = [synth.image(w, h, 3, rects=12, seed=60 + k) for k, (w, h) in enumerate(sizes)]
    imgs[1] = rng.random((3, 2003, 2111), dtype=np.float32)        # sparse: overflows once
    ss, sr = [12.0, 2.0, 16.0], [0.1, 0.05, 0.12]
    results = []
    for rep in range(2):   # the first call meets the noisy image's shape for the first time
        keep = [torch.from_numpy(im.copy()).pin_memory() for im in imgs]
        gpu.bilateral_batch([t.numpy() for t in keep], ss, sr)
        results.append([t.numpy().copy() for t in keep])
    expect = []
    for im, s, r in zip(imgs, ss, sr):
        e = im.copy()
        gpu.Bilateral.apply(e, s, s, 0.0, r)
        expect.append(e)
    for work in results:
        for w, e in zip(work, expect):
            assert rel_err(w, e) <= RTOL_FP32
