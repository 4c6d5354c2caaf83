"""B200 permutohedral-lattice Gauss transform, behind ImageStack's operation interface.

The compute path is ``libpermgpu.so`` (hand-written sm_100a kernels behind the C ABI of
``include/permgpu.h``), called through ctypes.  This module mirrors the reference's
static ``apply`` functions (src/GaussTransform.h:6-36) for the ``permutohedral_gpu``
method:

* ``GaussTransform.apply(slice, splat, values, sigmas)`` — un-normalised transform
  (src/GaussTransform.cpp:115-226);
* ``JointBilateral.apply(image, reference, fw, fh, ft, color_sigma)`` — in place
  (src/GaussTransform.cpp:504-678);
* ``Bilateral.apply(image, fw, fh, ft, color_sigma)`` — in place (:730-734).

Images are planar float32 arrays shaped (channels, frames, height, width) or
(channels, height, width): numpy arrays live in host memory; torch CUDA tensors are used
in place on the device.  There is no CPU path: without the library or a B200 every call
raises ``PgpuError``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpermgpu.so")

OK = 0
ERR_ARGUMENT, ERR_UNSUPPORTED, ERR_CUDA, ERR_MEMORY, ERR_CAPACITY = 1, 2, 3, 4, 5
ERR_NO_DEVICE, ERR_ADMISSION, ERR_TIMEOUT = 7, 8, 9

PAYLOADS = {"fp32": 0, "fp16": 1, "bf16": 2, "fp64": 3}
MEM_HOST, MEM_DEVICE = 0, 1


class PgpuError(RuntimeError):
    """A failed call into libpermgpu (the reference raises ImageStack::Exception)."""

    def __init__(self, code: int, message: str):
        super().__init__("permgpu error %d: %s" % (code, message))
        self.code = code


class Image(C.Structure):
    """pgpu_image: mirrors ImageStack::Image (src/Image.h:26-27)."""
    _fields_ = [("base", C.c_void_p), ("width", C.c_int), ("height", C.c_int),
                ("frames", C.c_int), ("channels", C.c_int), ("ystride", C.c_longlong),
                ("tstride", C.c_longlong), ("cstride", C.c_longlong)]


class Options(C.Structure):
    _fields_ = [("payload", C.c_int), ("memory", C.c_int), ("device", C.c_int),
                ("stream", C.c_void_p), ("load_factor", C.c_float), ("flags", C.c_int),
                ("method", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("points", C.c_longlong), ("vertices", C.c_longlong), ("capacity", C.c_longlong),
                ("d", C.c_int), ("vd", C.c_int), ("payload", C.c_int), ("retries", C.c_int),
                ("ms_splat", C.c_float), ("ms_compact", C.c_float), ("ms_neighbours", C.c_float),
                ("ms_blur", C.c_float), ("ms_slice", C.c_float), ("ms_total", C.c_float),
                ("load_factor", C.c_float), ("blur_pairs", C.c_int), ("tiled", C.c_int),
                ("blur_grid", C.c_int), ("tuned", C.c_int), ("nbr_half", C.c_int),
                ("vertex_rows", C.c_int), ("tile_w", C.c_int)]


from .tmpfile import load_tmp, save_tmp  # noqa: E402,F401  (ImageStack .tmp files)

EXPORTS = ["pgpu_default_options", "pgpu_last_error", "pgpu_version", "pgpu_device_count",
           "pgpu_gauss_transform", "pgpu_joint_bilateral", "pgpu_bilateral", "pgpu_last_stats",
           "pgpu_lattice_dump", "pgpu_bilateral_batch", "pgpu_exact_gauss_transform_f64",
           "pgpu_probe_red_rate", "pgpu_bilateral_batch_submit", "pgpu_batch_wait"]

_lib = None


def lib():
    """Load libpermgpu.so (raises PgpuError if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PgpuError(ERR_NO_DEVICE, "libpermgpu.so is not built (python -m imagestack_b200.build)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    L.pgpu_default_options.argtypes = [P(Options)]
    L.pgpu_last_error.restype = C.c_char_p
    L.pgpu_gauss_transform.argtypes = [P(Image), P(Image), P(Image), P(C.c_float), C.c_int,
                                       P(Image), P(Options)]
    L.pgpu_joint_bilateral.argtypes = [P(Image), P(Image), C.c_float, C.c_float, C.c_float,
                                       C.c_float, P(Options)]
    L.pgpu_bilateral.argtypes = [P(Image), C.c_float, C.c_float, C.c_float, C.c_float, P(Options)]
    L.pgpu_last_stats.argtypes = [P(Stats)]
    L.pgpu_bilateral_batch.argtypes = [P(Image), C.c_int, P(C.c_float), P(C.c_float), P(Options)]
    L.pgpu_bilateral_batch_submit.argtypes = [P(Image), P(Image), C.c_int, P(C.c_float), P(C.c_float),
                                              P(Options), P(C.c_longlong)]
    L.pgpu_batch_wait.argtypes = [C.c_longlong]
    L.pgpu_lattice_dump.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                    P(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p]
    L.pgpu_exact_gauss_transform_f64.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.pgpu_probe_red_rate.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_void_p,
                                      C.POINTER(C.c_double)]
    _lib = L
    return L


def _check(rc: int):
    if rc != OK:
        raise PgpuError(rc, lib().pgpu_last_error().decode(errors="replace"))


def exact_gauss_transform_f64(queries, positions, values):
    """FP64 brute-force Gauss transform on the GPU: for each query row,
    sum_j exp(-|q - p_j|^2 / 2) v_j over all rows of `positions` (already divided by the
    sigmas), as the EXACT method of GaussTransform::apply (src/GaussTransform.cpp:135-162)
    defines it but with an exact exponential.  CUDA float32 tensors, interleaved
    (queries nq x d, positions n x d, values n x vd); returns an nq x vd float64 tensor.
    It states the error of lattice results and is not a filtering path."""
    import torch
    q = queries.contiguous()
    p = positions.contiguous()
    v = values.contiguous()
    for t in (q, p, v):
        if not (t.is_cuda and t.dtype == torch.float32 and t.dim() == 2):
            raise PgpuError(ERR_ARGUMENT, "CUDA float32 matrices expected")
    if q.shape[1] != p.shape[1] or p.shape[0] != v.shape[0]:
        raise PgpuError(ERR_ARGUMENT, "mismatched shapes")
    out = torch.empty((q.shape[0], v.shape[1]), dtype=torch.float64, device=q.device)
    stream = C.c_void_p(torch.cuda.current_stream(q.device).cuda_stream)
    _check(lib().pgpu_exact_gauss_transform_f64(q.shape[1], v.shape[1], q.shape[0], q.data_ptr(),
                                                p.shape[0], p.data_ptr(), v.data_ptr(),
                                                out.data_ptr(), stream))
    return out


def probe_red_rate(rows: int, per_thread: int = 64, blocks: int | None = None) -> float:
    """Float4 reductions per second this GPU retires at pseudo-random rows of a table of
    `rows` x 16 bytes (the splat's atomic access); the splat's roofline for atomics."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    table = torch.zeros((rows, 4), dtype=torch.float32, device=dev)
    if blocks is None:
        blocks = 8 * torch.cuda.get_device_properties(dev).multi_processor_count
    out = C.c_double(0.0)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _check(lib().pgpu_probe_red_rate(table.data_ptr(), rows, per_thread, blocks, stream,
                                     C.byref(out)))
    return out.value


def last_stats() -> dict:
    s = Stats()
    _check(lib().pgpu_last_stats(C.byref(s)))
    return {k: getattr(s, k) for k, _ in Stats._fields_}


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _view(a, name: str) -> tuple[Image, int]:
    """pgpu_image of a planar (c, f, h, w) / (c, h, w) float32 array; returns (view, memory)."""
    if _is_torch(a):
        import torch
        if a.dtype != torch.float32:
            raise PgpuError(ERR_ARGUMENT, "%s must be float32" % name)
        t = a if a.dim() == 4 else a.unsqueeze(1)
        if t.dim() != 4 or t.stride(3) != 1:
            raise PgpuError(ERR_ARGUMENT, "%s must be (c, [f,] h, w) with unit x stride" % name)
        c, f, h, w = t.shape
        v = Image(t.data_ptr(), w, h, f, c, t.stride(2), t.stride(1), t.stride(0))
        return v, (MEM_DEVICE if t.is_cuda else MEM_HOST)
    if not isinstance(a, np.ndarray) or a.dtype != np.float32:
        raise PgpuError(ERR_ARGUMENT, "%s must be a float32 numpy array or torch tensor" % name)
    t = a if a.ndim == 4 else a[:, None]
    if t.ndim != 4 or t.strides[3] != 4:
        raise PgpuError(ERR_ARGUMENT, "%s must be (c, [f,] h, w) with unit x stride" % name)
    c, f, h, w = t.shape
    s = [x // 4 for x in t.strides]
    v = Image(t.ctypes.data, w, h, f, c, s[2], s[1], s[0])
    return v, MEM_HOST


_IMAGE_DTYPE = np.dtype([("base", np.uintp), ("width", np.int32), ("height", np.int32),
                         ("frames", np.int32), ("channels", np.int32), ("ystride", np.int64),
                         ("tstride", np.int64), ("cstride", np.int64)])
assert _IMAGE_DTYPE.itemsize == C.sizeof(Image)


def _views_torch(images):
    """Views of many torch tensors at once: one column per pgpu_image field, filled by
    list comprehensions into a buffer laid out like the C array (a per-image ctypes
    structure costs several microseconds).  Returns (views, memory), or None when any
    image would fail _view's checks, so that the per-image path raises its message."""
    import torch
    try:
        dims = [a.dim() for a in images]
        if any(a.dtype != torch.float32 for a in images):
            return None
        cuda = [a.is_cuda for a in images]
    except AttributeError:
        return None
    if not (all(cuda) or not any(cuda)) or any(k not in (3, 4) for k in dims):
        return None
    shapes = [a.shape for a in images]
    strides = [a.stride() for a in images]
    if any(s[-1] != 1 for s in strides):
        return None
    n = len(images)
    arr = np.empty(n, _IMAGE_DTYPE)
    arr["base"] = [a.data_ptr() for a in images]
    arr["channels"] = [s[0] for s in shapes]
    arr["width"] = [s[-1] for s in shapes]
    arr["height"] = [s[-2] for s in shapes]
    arr["frames"] = [s[1] if k == 4 else 1 for s, k in zip(shapes, dims)]
    arr["ystride"] = [s[-2] for s in strides]
    arr["cstride"] = [s[0] for s in strides]
    # A (c, h, w) tensor is the single frame of (c, 1, h, w), whose frame stride torch's
    # unsqueeze(1) sets to height x row stride.
    arr["tstride"] = [s[1] if k == 4 else s[1] * sh[1]
                      for s, sh, k in zip(strides, shapes, dims)]
    views = (Image * n).from_buffer(arr)
    return views, (MEM_DEVICE if cuda[0] else MEM_HOST)


def _options(memory: int, payload: str, device: int = 0, stream=None, load_factor: float = 0.5):
    o = Options()
    lib().pgpu_default_options(C.byref(o))
    o.payload = PAYLOADS[payload]
    o.memory = memory
    o.device = device
    o.stream = stream
    o.load_factor = load_factor
    return o


def _torch_stream(a):
    import torch
    return C.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)


METHODS = {"permutohedral_gpu": 0, "grid_gpu": 1}   # PGPU_METHOD_PERMUTOHEDRAL, _GRID


def _method_ok(method: str) -> int:
    """The library's method code for a method token: permutohedral_gpu (the lattice) or
    grid_gpu (the bilateral grid); the reference's other methods stay on its CPU path."""
    if method not in METHODS:
        raise PgpuError(ERR_UNSUPPORTED,
                        "methods here: permutohedral_gpu, grid_gpu; the reference's other "
                        "methods stay on its CPU path")
    return METHODS[method]


class GaussTransform:
    """GaussTransform::apply with the permutohedral_gpu method."""

    @staticmethod
    def apply(slice_positions, splat_positions, values, sigmas, method: str = "permutohedral_gpu",
              payload: str = "fp32", load_factor: float = 0.5):
        mcode = _method_ok(method)
        same = slice_positions is None or slice_positions is splat_positions
        sp, mem = _view(splat_positions, "splat")
        va, mem2 = _view(values, "values")
        sl = sp if same else _view(slice_positions, "slice")[0]
        if mem != mem2:
            raise PgpuError(ERR_ARGUMENT, "images must all be on the host or all on the device")
        src = splat_positions if same else slice_positions
        shape = (values.shape[0],) + tuple(src.shape[1:])
        if _is_torch(splat_positions):
            import torch
            out = torch.empty(shape, dtype=torch.float32, device=splat_positions.device)
        else:
            out = np.empty(shape, np.float32)
        ov, _ = _view(out, "out")
        sig = (C.c_float * len(sigmas))(*[float(s) for s in sigmas])
        stream = _torch_stream(splat_positions) if mem == MEM_DEVICE else None
        opt = _options(mem, payload, stream=stream, load_factor=load_factor,
                       device=(splat_positions.device.index or 0) if mem == MEM_DEVICE else 0)
        opt.method = mcode
        _check(lib().pgpu_gauss_transform(None if same else C.byref(sl), C.byref(sp), C.byref(va),
                                          sig, len(sigmas), C.byref(ov), C.byref(opt)))
        return out


class JointBilateral:
    """JointBilateral::apply with the permutohedral_gpu method (in place on `image`)."""

    @staticmethod
    def apply(image, reference, filter_width: float, filter_height: float, filter_frames: float,
              color_sigma: float, method: str = "permutohedral_gpu", payload: str = "fp32",
              load_factor: float = 0.5):
        mcode = _method_ok(method)
        im, mem = _view(image, "image")
        ref, mem2 = _view(reference, "reference")
        if mem != mem2:
            raise PgpuError(ERR_ARGUMENT, "image and reference must be in the same memory")
        stream = _torch_stream(image) if mem == MEM_DEVICE else None
        opt = _options(mem, payload, stream=stream, load_factor=load_factor,
                       device=(image.device.index or 0) if mem == MEM_DEVICE else 0)
        opt.method = mcode
        _check(lib().pgpu_joint_bilateral(C.byref(im), C.byref(ref), filter_width, filter_height,
                                          filter_frames, color_sigma, C.byref(opt)))
        return image


class Bilateral:
    """Bilateral::apply with the permutohedral_gpu method (in place)."""

    @staticmethod
    def apply(image, filter_width: float, filter_height: float, filter_frames: float,
              color_sigma: float, method: str = "permutohedral_gpu", payload: str = "fp32",
              load_factor: float = 0.5):
        mcode = _method_ok(method)
        im, mem = _view(image, "image")
        stream = _torch_stream(image) if mem == MEM_DEVICE else None
        opt = _options(mem, payload, stream=stream, load_factor=load_factor,
                       device=(image.device.index or 0) if mem == MEM_DEVICE else 0)
        opt.method = mcode
        _check(lib().pgpu_bilateral(C.byref(im), filter_width, filter_height, filter_frames,
                                    color_sigma, C.byref(opt)))
        return image


FLAG_GRAPH = 1
FLAG_AUTOTUNE = 2


def bilateral_batch(images, filter_widths, color_sigmas, payload: str = "fp32",
                    graph: bool = False, load_factor: float = 0.5, autotune: bool = False):
    """Bilateral filter of many images (same channel count, any sizes) in one set of
    launches, each in place with its own sigmas; the result of each equals
    Bilateral.apply on it.  All numpy (host) or all torch CUDA tensors (device, run on
    torch's current stream).  graph: capture the launches as a CUDA graph and replay it
    for later batches of the same shape.  autotune: the first calls of each batch shape
    try candidate load factors and blur pairings, later calls use the fastest."""
    n = len(images)
    if len(filter_widths) != n or len(color_sigmas) != n:
        raise PgpuError(ERR_ARGUMENT, "one filter width and colour sigma per image")
    fast = _views_torch(images) if n and _is_torch(images[0]) else None
    if fast is not None:
        views, mem = fast
    else:
        views = (Image * max(n, 1))()
        mem = MEM_HOST
        for i, im in enumerate(images):
            views[i], m = _view(im, "image %d" % i)
            if i == 0:
                mem = m
            elif m != mem:
                raise PgpuError(ERR_ARGUMENT, "images must all be on the host or all on the device")
    fw = (C.c_float * max(n, 1))(*[float(x) for x in filter_widths])
    cs = (C.c_float * max(n, 1))(*[float(x) for x in color_sigmas])
    stream = _torch_stream(images[0]) if (n and mem == MEM_DEVICE) else None
    opt = _options(mem, payload, stream=stream, load_factor=load_factor,
                   device=(images[0].device.index or 0) if (n and mem == MEM_DEVICE) else 0)
    opt.flags = (FLAG_GRAPH if graph else 0) | (FLAG_AUTOTUNE if autotune else 0)
    _check(lib().pgpu_bilateral_batch(views, n, fw, cs, C.byref(opt)))
    return images


class BatchTicket:
    """A host batch queued by bilateral_batch_submit.  wait() returns the outputs once
    they are written; the input and output arrays are held (and must not be modified)
    until then.  A ticket dropped without wait() is waited for first."""

    def __init__(self, ticket: int, images, outputs):
        self.ticket = ticket
        self.images = images
        self.outputs = outputs
        self.done = False

    def wait(self):
        if not self.done:
            self.done = True
            _check(lib().pgpu_batch_wait(self.ticket))
        return self.outputs

    def __del__(self):
        if not getattr(self, "done", True):
            try:
                self.wait()
            except Exception:
                pass


def bilateral_batch_submit(images, filter_widths, color_sigmas, outputs=None, payload: str = "fp32",
                           graph: bool = False, load_factor: float = 0.5, autotune: bool = False):
    """Queue the bilateral filter of many host (numpy) images and return a BatchTicket at
    once (pgpu_bilateral_batch_submit): each result goes to outputs[i] (same shape; None:
    in place).  Consecutive submissions overlap their copies and filtering on the device;
    each result equals Bilateral.apply on the image."""
    n = len(images)
    if n == 0 or len(filter_widths) != n or len(color_sigmas) != n:
        raise PgpuError(ERR_ARGUMENT, "one filter width and colour sigma per image, at least one image")
    if outputs is not None and len(outputs) != n:
        raise PgpuError(ERR_ARGUMENT, "one output per image")
    views = (Image * n)()
    outs = (Image * n)() if outputs is not None else None
    for i, im in enumerate(images):
        views[i], m = _view(im, "image %d" % i)
        if m != MEM_HOST:
            raise PgpuError(ERR_ARGUMENT, "queued batches take host (numpy) images")
        if outs is not None:
            outs[i], m = _view(outputs[i], "output %d" % i)
            if m != MEM_HOST:
                raise PgpuError(ERR_ARGUMENT, "queued batches take host (numpy) outputs")
    fw = (C.c_float * n)(*[float(x) for x in filter_widths])
    cs = (C.c_float * n)(*[float(x) for x in color_sigmas])
    opt = _options(MEM_HOST, payload, load_factor=load_factor)
    opt.flags = (FLAG_GRAPH if graph else 0) | (FLAG_AUTOTUNE if autotune else 0)
    t = C.c_longlong(0)
    _check(lib().pgpu_bilateral_batch_submit(views, outs, n, fw, cs, C.byref(opt), C.byref(t)))
    return BatchTicket(t.value, images, outputs if outputs is not None else images)


REQ_BILATERAL, REQ_JOINT_BILATERAL, REQ_GAUSS_TRANSFORM = 0, 1, 2


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("workers", C.c_int), ("max_batch", C.c_int),
                ("payload", C.c_int), ("load_factor", C.c_float), ("memory_budget", C.c_longlong)]


class Request(C.Structure):
    _fields_ = [("kind", C.c_int), ("in_", Image), ("ref", Image), ("out", Image),
                ("filter_width", C.c_float), ("color_sigma", C.c_float),
                ("sigmas", C.POINTER(C.c_float)), ("n_sigmas", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_longlong) for k in ("submitted", "completed", "failed", "rejected", "queued",
                                             "in_flight", "batches", "pixels", "peak_bytes")] + \
               [(k, C.c_double) for k in ("seconds", "p50_ms", "p99_ms", "mean_ms", "max_ms",
                                          "mpix_per_s", "req_per_s")]


class Server:
    """Continuous-batching request server (pgpu_server_*): host images in, results written
    to each request's output array.  Requests of different sizes and kinds are batched as
    they arrive and run on several device streams at once."""

    def __init__(self, workers: int = 2, max_batch: int = 64, payload: str = "fp32",
                 memory_budget: int = 40 << 30, device: int = 0, load_factor: float = 0.5):
        L = lib()
        L.pgpu_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]
        L.pgpu_server_submit.argtypes = [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_longlong)]
        L.pgpu_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_int]
        L.pgpu_server_drain.argtypes = [C.c_void_p, C.c_int]
        L.pgpu_server_get_stats.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        L.pgpu_server_reset_stats.argtypes = [C.c_void_p]
        L.pgpu_server_destroy.argtypes = [C.c_void_p]
        cfg = ServerConfig(device, workers, max_batch, PAYLOADS[payload], load_factor, memory_budget)
        h = C.c_void_p()
        _check(L.pgpu_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, kind: int, image, out, ref=None, filter_width: float = 0.0,
               color_sigma: float = 0.0, sigmas=None) -> int:
        """Queue a request; the arrays must stay alive until wait() returns for it."""
        r = Request()
        r.kind = kind
        r.in_ = _view(image, "image")[0]
        r.out = _view(out, "out")[0]
        if ref is not None:
            r.ref = _view(ref, "ref")[0]
        r.filter_width = filter_width
        r.color_sigma = color_sigma
        sig = None
        if sigmas is not None:
            sig = (C.c_float * len(sigmas))(*[float(s) for s in sigmas])
            r.sigmas = C.cast(sig, C.POINTER(C.c_float))
            r.n_sigmas = len(sigmas)
        t = C.c_longlong()
        _check(lib().pgpu_server_submit(self._h, C.byref(r), C.byref(t)))
        self._keep[t.value] = (image, out, ref, sig)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 600000):
        rc = lib().pgpu_server_wait(self._h, ticket, timeout_ms)
        if rc != ERR_TIMEOUT:
            self._keep.pop(ticket, None)
        _check(rc)

    def drain(self, timeout_ms: int = 600000):
        _check(lib().pgpu_server_drain(self._h, timeout_ms))

    def stats(self) -> dict:
        s = ServerStats()
        _check(lib().pgpu_server_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def reset_stats(self):
        _check(lib().pgpu_server_reset_stats(self._h))

    def close(self):
        if self._h:
            lib().pgpu_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def lattice_dump(pos: np.ndarray, val: np.ndarray, payload: str = "fp32") -> dict:
    """Everything one lattice computes for n interleaved points (pos scaled by 1/sigma):
    keys (M, d) in vertex order, replay vertex index and weight (n, d+1), vertex values
    after splat and after blur (M, vd), and the replay slice (n, vd)."""
    pos = np.ascontiguousarray(pos, np.float32)
    val = np.ascontiguousarray(val, np.float32)
    n, d = pos.shape
    vd = val.shape[1]
    rows = n * (d + 1)
    m = C.c_int(0)
    keys = np.empty((rows, d), np.int16)
    rv = np.empty((n, d + 1), np.int32)
    rw = np.empty((n, d + 1), np.float32)
    sv = np.empty((rows, vd), np.float32)
    bv = np.empty((rows, vd), np.float32)
    out = np.empty((n, vd), np.float32)
    _check(lib().pgpu_lattice_dump(d, vd, n, pos.ctypes.data, val.ctypes.data, PAYLOADS[payload],
                                   C.byref(m), keys.ctypes.data, rv.ctypes.data, rw.ctypes.data,
                                   sv.ctypes.data, bv.ctypes.data, out.ctypes.data))
    M = m.value
    return {"keys": keys[:M].copy(), "replay_vtx": rv, "replay_w": rw, "splat": sv[:M].copy(),
            "blur": bv[:M].copy(), "out": out}


def device_count() -> int:
    return int(lib().pgpu_device_count())
