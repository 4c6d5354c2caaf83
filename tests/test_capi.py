"""The C-ABI library without a GPU: it loads, exports every declared entry point, and
fails loudly (never silently on a CPU path) when no B200 is present."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import imagestack_b200 as ib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b(pgpu_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_entry_point():
    lib = C.CDLL(ib.LIB_PATH)
    names = declared_functions()
    assert "pgpu_bilateral" in names and "pgpu_gauss_transform" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_entry_point():
    for n in declared_functions():
        assert n in ib.EXPORTS or n.startswith("pgpu_server") or n.startswith("pgpu_batch") \
            or n.startswith("pgpu_lattice") or n.startswith("pgpu_bilateral_noalloc"), n


def test_default_options_and_version():
    o = ib.Options()
    ib.lib().pgpu_default_options(C.byref(o))
    assert o.payload == 0 and o.memory == 0 and abs(o.load_factor - 0.5) < 1e-7
    assert ib.lib().pgpu_version() >= 100


def _has_device():
    return ib.device_count() > 0


@pytest.mark.skipif(_has_device(), reason="checks the no-GPU behaviour")
def test_no_device_fails_loudly():
    img = np.random.default_rng(0).random((3, 16, 16), dtype=np.float32)
    with pytest.raises(ib.PgpuError) as e:
        ib.Bilateral.apply(img, 4.0, 4.0, 0.0, 0.1)
    assert e.value.code == ib.ERR_NO_DEVICE
    with pytest.raises(ib.PgpuError) as e:
        ib.bilateral_batch_submit([img], [4.0], [0.1])
    assert e.value.code == ib.ERR_NO_DEVICE


def test_other_methods_are_not_served_here():
    img = np.zeros((3, 8, 8), np.float32)
    with pytest.raises(ib.PgpuError) as e:
        ib.Bilateral.apply(img, 4.0, 4.0, 0.0, 0.1, method="permutohedral")
    assert e.value.code == ib.ERR_UNSUPPORTED


def test_views_mirror_image_addressing():
    a = np.zeros((4, 2, 5, 7), np.float32)   # (c, f, h, w)
    v, mem = ib._view(a, "a")
    assert mem == ib.MEM_HOST
    assert (v.width, v.height, v.frames, v.channels) == (7, 5, 2, 4)
    assert (v.ystride, v.tstride, v.cstride) == (7, 35, 70)
    sub = a[1:3, :, 1:4, 2:6]                # a region view shares the payload
    v, _ = ib._view(sub, "sub")
    assert (v.width, v.height, v.frames, v.channels) == (4, 3, 2, 2)
    assert (v.ystride, v.tstride, v.cstride) == (7, 35, 70)
    with pytest.raises(ib.PgpuError):
        ib._view(a.astype(np.float64), "f64")


def test_views_beyond_the_point_numbering_are_refused_before_any_device_work():
    """A lattice numbers its points in 32 bits: a view of 65536 x 65536 pixels (2^32
    points) is refused with ERR_UNSUPPORTED by every entry point, before the library
    looks for a device or reads a pixel (the base address is never dereferenced)."""
    lib = ib.lib()
    buf = np.zeros(16, np.float32)
    n = 1 << 16
    big = ib.Image(buf.ctypes.data, n, n, 1, 3, n, n * n, n * n)
    small = ib.Image(buf.ctypes.data, 4, 4, 1, 3, 4, 16, 16)
    opt = ib.Options()
    lib.pgpu_default_options(C.byref(opt))
    rc = lib.pgpu_joint_bilateral(C.byref(big), C.byref(big), 8.0, 8.0, 0.0, 0.1, C.byref(opt))
    assert rc == ib.ERR_UNSUPPORTED and b"2^32" in lib.pgpu_last_error()
    sig = (C.c_float * 3)(1.0, 1.0, 1.0)
    rc = lib.pgpu_gauss_transform(None, C.byref(big), C.byref(big), sig, 3, C.byref(big), C.byref(opt))
    assert rc == ib.ERR_UNSUPPORTED
    rc = lib.pgpu_gauss_transform(C.byref(big), C.byref(small), C.byref(small), sig, 3, C.byref(big),
                                  C.byref(opt))
    assert rc == ib.ERR_UNSUPPORTED
    fw, cs = (C.c_float * 1)(8.0), (C.c_float * 1)(0.1)
    assert lib.pgpu_bilateral_batch(C.byref(big), 1, fw, cs, C.byref(opt)) == ib.ERR_UNSUPPORTED
    ticket = C.c_longlong(0)
    rc = lib.pgpu_bilateral_batch_submit(C.byref(big), None, 1, fw, cs, C.byref(opt), C.byref(ticket))
    assert rc == ib.ERR_UNSUPPORTED and ticket.value == 0
