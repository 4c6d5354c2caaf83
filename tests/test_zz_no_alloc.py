"""pgpu_bilateral_noalloc: the entry point for callers that cannot allocate device memory
(hosts that own every byte through their own pool, or loops that must not let
cudaMalloc/cudaFree synchronise the device).  It keeps all intermediates in a fixed array
inside the library; this checks, through the C ABI, that two calls in a row (the second
reusing the array the first left behind) match pgpu_bilateral within the tolerance of the
other parity tests, and that oversized requests are refused.

The file name sorts last so that a run stopping at its first failure has already run every
other test; the test passes alone in a fresh process as well as after the others.
"""
import ctypes as C

import numpy as np
import pytest

from imagestack_b200 import synth

pytestmark = pytest.mark.gpu

RTOL_FP32 = 1e-5


def rel_err(a, b, floor_frac=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    floor = max(np.abs(b).max() * floor_frac, 1e-30)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max())


def _noalloc(gpu):
    f = gpu.lib().pgpu_bilateral_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                  C.c_float, C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_matches_bilateral_on_two_calls_in_a_row(gpu):
    import torch
    noalloc = _noalloc(gpu)
    stream = torch.cuda.current_stream().cuda_stream
    # the second call is smaller and has fewer channels, so leftovers of the first call in
    # the shared array would show
    cases = [(512, 512, 3, 8.0, 0.1, 31), (300, 200, 1, 5.0, 0.2, 32)]
    for w, h, c, ss, sr, seed in cases:
        img = synth.image(w, h, c, rects=10, seed=seed)
        expect = torch.from_numpy(img.copy()).cuda()
        gpu.Bilateral.apply(expect, ss, ss, 0.0, sr)            # the existing entry point
        src = torch.from_numpy(img).cuda()
        out = torch.full_like(src, float("nan"))
        torch.cuda.synchronize()
        rc = noalloc(src.data_ptr(), out.data_ptr(), w, h, c, ss, ss, sr, stream)
        assert rc == 0, gpu.lib().pgpu_last_error().decode()
        torch.cuda.synchronize()
        assert rel_err(out.cpu().numpy(), expect.cpu().numpy()) <= RTOL_FP32
        np.testing.assert_array_equal(src.cpu().numpy(), img)   # input untouched


def test_noalloc_refuses_sizes_beyond_its_array(gpu):
    import torch
    noalloc = _noalloc(gpu)
    big = torch.zeros((3, 600, 600), device="cuda")
    rc = noalloc(big.data_ptr(), big.data_ptr(), 600, 600, 3, 8.0, 8.0, 0.1, None)
    assert rc == gpu.ERR_UNSUPPORTED
    assert b"262144" in gpu.lib().pgpu_last_error()
    four = torch.zeros((4, 64, 64), device="cuda")
    assert noalloc(four.data_ptr(), four.data_ptr(), 64, 64, 4, 8.0, 8.0, 0.1, None) == \
        gpu.ERR_UNSUPPORTED


def test_noalloc_overfull_lattice_leaves_output_unwritten_and_recovers(gpu):
    """A frame inside the size limits whose lattice still needs more hash slots than the
    array holds (uniform noise with small sigmas: almost every (pixel, remainder) is its own
    vertex) is refused with ERR_CAPACITY and d_out is left as it was; the next call starts
    from a clean array and matches pgpu_bilateral again."""
    import torch
    noalloc = _noalloc(gpu)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    noise = torch.from_numpy(rng.random((3, 512, 512), dtype=np.float32)).cuda()
    out = torch.full_like(noise, float("nan"))
    torch.cuda.synchronize()
    rc = noalloc(noise.data_ptr(), out.data_ptr(), 512, 512, 3, 1.0, 1.0, 0.02, stream)
    torch.cuda.synchronize()
    assert rc == gpu.ERR_CAPACITY, gpu.lib().pgpu_last_error().decode()
    assert torch.isnan(out).all().item()
    img = synth.image(256, 256, 3, rects=8, seed=33)
    expect = torch.from_numpy(img.copy()).cuda()
    gpu.Bilateral.apply(expect, 8.0, 8.0, 0.0, 0.1)
    src = torch.from_numpy(img).cuda()
    out2 = torch.full_like(src, float("nan"))
    torch.cuda.synchronize()
    assert noalloc(src.data_ptr(), out2.data_ptr(), 256, 256, 3, 8.0, 8.0, 0.1, stream) == 0
    torch.cuda.synchronize()
    assert rel_err(out2.cpu().numpy(), expect.cpu().numpy()) <= RTOL_FP32


def test_noalloc_refuses_to_run_inside_a_stream_capture(gpu):
    """A call waits for its stream, so it cannot be part of a CUDA graph: during a capture
    it returns ERR_UNSUPPORTED and queues nothing."""
    import torch
    noalloc = _noalloc(gpu)
    img = torch.zeros((1, 64, 64), device="cuda")
    out = torch.zeros_like(img)
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=side):
        out.add_(1.0)   # the graph needs one node of its own
        rc = noalloc(img.data_ptr(), out.data_ptr(), 64, 64, 1, 4.0, 4.0, 0.1,
                     torch.cuda.current_stream().cuda_stream)
    assert rc == gpu.ERR_UNSUPPORTED
    assert b"capture" in gpu.lib().pgpu_last_error()
    g.replay()
    torch.cuda.synchronize()
    assert (out == 1.0).all().item()
