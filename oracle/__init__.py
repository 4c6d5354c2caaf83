"""CPU checkers for the permutohedral lattice — TEST INFRASTRUCTURE, not the product.

Two checkers live here, loaded through ctypes:

* ``liblattice_oracle.so`` — my plain-C restatement of src/Permutohedral.h
  (oracle/lattice_oracle.c): FP32 mode bit-exact with the reference, FP64-accumulation
  mode (the FP64 lattice oracle), and an FP64 brute-force Gauss transform.
* ``_ref/libref_harness.so`` — the reference ImageStack compiled from its own sources
  with strict IEEE flags (oracle/Makefile), driven by oracle/ref_harness.cpp.  Present
  wherever it was built; tests that need it skip when it is absent.

Only tests/, the smoke check and the benchmark's CPU-baseline leg import this package.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liblattice_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_HARNESS_SO = os.path.join(REF_DIR, "libref_harness.so")
# the same harness over the reference built with its shipped flags (-ffast-math); for
# timing only, loaded instead of the strict one when PGPU_REFERENCE_BUILD=shipped
REF_HARNESS_FAST_SO = os.path.join(REF_DIR, "libref_harness_fast.so")
REF_CLI = os.path.join(REF_DIR, "ImageStack")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i16p = np.ctypeslib.ndpointer(np.int16, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")

METHODS = {"auto": 0, "exact": 1, "grid": 2, "permutohedral": 3, "gkdtree": 4}

_lo = None
_ref = None


def _load_oracle():
    global _lo
    if _lo is None:
        lib = C.CDLL(ORACLE_SO)
        lib.lo_scale_factors.argtypes = [C.c_int, _f32p]
        lib.lo_simplex.argtypes = [C.c_int, C.c_int, _f32p, _i16p, _f32p]
        lib.lo_create.restype = C.c_void_p
        lib.lo_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
        lib.lo_destroy.argtypes = [C.c_void_p]
        lib.lo_splat.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int]
        lib.lo_size.argtypes = [C.c_void_p]
        lib.lo_keys.argtypes = [C.c_void_p, _i16p]
        lib.lo_values_f32.argtypes = [C.c_void_p, _f32p]
        lib.lo_values_f64.argtypes = [C.c_void_p, _f64p]
        lib.lo_replay.argtypes = [C.c_void_p, _i32p, _f32p]
        lib.lo_blur.argtypes = [C.c_void_p]
        lib.lo_slice_replay_f32.argtypes = [C.c_void_p, _f32p]
        lib.lo_slice_replay_f64.argtypes = [C.c_void_p, _f64p]
        lib.lo_slice_positions_f32.argtypes = [C.c_void_p, _f32p, C.c_int, _f32p]
        lib.lo_slice_positions_f64.argtypes = [C.c_void_p, _f32p, C.c_int, _f64p]
        lib.lo_exact_gt_f64.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, C.c_int, _f32p,
                                        _f32p, _f64p]
        _lo = lib
    return _lo


def _harness_path() -> str:
    return REF_HARNESS_FAST_SO if os.environ.get("PGPU_REFERENCE_BUILD") == "shipped" else REF_HARNESS_SO


def reference_available() -> bool:
    return os.path.exists(_harness_path())


def _load_ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(_harness_path())
        lib.refh_last_error.restype = C.c_char_p
        lib.refh_lattice_create.restype = C.c_void_p
        lib.refh_lattice_create.argtypes = [C.c_int, C.c_int, C.c_int]
        lib.refh_lattice_destroy.argtypes = [C.c_void_p]
        lib.refh_lattice_splat.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int]
        lib.refh_lattice_size.argtypes = [C.c_void_p]
        lib.refh_lattice_keys.argtypes = [C.c_void_p, _i16p]
        lib.refh_lattice_values.argtypes = [C.c_void_p, _f32p]
        lib.refh_lattice_replay.argtypes = [C.c_void_p, _i32p, _f32p]
        lib.refh_lattice_blur.argtypes = [C.c_void_p]
        lib.refh_lattice_slice_replay.argtypes = [C.c_void_p, _f32p, C.c_int]
        lib.refh_lattice_slice_positions.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int]
        lib.refh_gauss_transform.restype = C.c_double
        lib.refh_gauss_transform.argtypes = [_f32p, _f32p, C.c_int, _f32p, C.c_int, C.c_int,
                                             C.c_int, C.c_int, C.c_int, _f32p, C.c_int, _f32p]
        lib.refh_joint_bilateral.restype = C.c_double
        lib.refh_joint_bilateral.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.c_int, C.c_float, C.c_float, C.c_float,
                                             C.c_float, C.c_int]
        lib.refh_bilateral.restype = C.c_double
        lib.refh_bilateral.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                       C.c_float, C.c_float, C.c_float, C.c_int]
        lib.refh_nlmeans3d.restype = C.c_double
        lib.refh_nlmeans3d.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_float, C.c_int, C.c_float, C.c_float, C.c_int]
        _ref = lib
    return _ref


@dataclass
class LatticeDump:
    """Everything the lattice computes for one set of points."""
    keys: np.ndarray          # (M, d) int16, vertex order = first insertion
    replay_vtx: np.ndarray    # (n, d+1) int32
    replay_w: np.ndarray      # (n, d+1) float32
    splat: np.ndarray         # (M, vd) values after splat
    blur: np.ndarray          # (M, vd) values after blur
    out: np.ndarray           # (n, vd) replay slice


def _check(pos: np.ndarray, val: np.ndarray):
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    val = np.ascontiguousarray(val, dtype=np.float32)
    assert pos.ndim == 2 and val.ndim == 2 and pos.shape[0] == val.shape[0]
    return pos, val


def oracle_lattice(pos: np.ndarray, val: np.ndarray, fp64: bool = False,
                   slice_pos: np.ndarray | None = None) -> LatticeDump:
    """Run the C restatement on interleaved points (pos already scaled by 1/sigma)."""
    lib = _load_oracle()
    pos, val = _check(pos, val)
    n, d = pos.shape
    vd = val.shape[1]
    h = lib.lo_create(d, vd, n, 1 if fp64 else 0)
    if not h:
        raise MemoryError("lo_create failed")
    try:
        rc = lib.lo_splat(h, pos, val, n)
        if rc == -2:
            raise ValueError("positions leave the lattice's int16 key range")
        if rc != 0:
            raise MemoryError("lo_splat failed")
        m = lib.lo_size(h)
        keys = np.empty((m, d), np.int16)
        lib.lo_keys(h, keys)
        rv = np.empty((n, d + 1), np.int32)
        rw = np.empty((n, d + 1), np.float32)
        lib.lo_replay(h, rv, rw)
        dt = np.float64 if fp64 else np.float32
        sp = np.empty((m, vd), dt)
        (lib.lo_values_f64 if fp64 else lib.lo_values_f32)(h, sp)
        lib.lo_blur(h)
        bl = np.empty((m, vd), dt)
        (lib.lo_values_f64 if fp64 else lib.lo_values_f32)(h, bl)
        if slice_pos is None:
            out = np.empty((n, vd), dt)
            (lib.lo_slice_replay_f64 if fp64 else lib.lo_slice_replay_f32)(h, out)
        else:
            sp_ = np.ascontiguousarray(slice_pos, dtype=np.float32)
            out = np.empty((sp_.shape[0], vd), dt)
            (lib.lo_slice_positions_f64 if fp64 else lib.lo_slice_positions_f32)(
                h, sp_, sp_.shape[0], out)
        return LatticeDump(keys, rv, rw, sp, bl, out)
    finally:
        lib.lo_destroy(h)


def oracle_simplex(pos: np.ndarray):
    """Per point: keys (n, d+1, d) int16 and barycentric weights (n, d+1) float32."""
    lib = _load_oracle()
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    n, d = pos.shape
    keys = np.empty((n, d + 1, d), np.int16)
    bary = np.empty((n, d + 1), np.float32)
    lib.lo_simplex(d, n, pos, keys, bary)
    return keys, bary


def exact_gauss_transform(query: np.ndarray, pos: np.ndarray, val: np.ndarray) -> np.ndarray:
    """FP64 brute force sum_j exp(-|q_i-p_j|^2/2) v_j for the given queries."""
    lib = _load_oracle()
    q = np.ascontiguousarray(query, dtype=np.float32)
    pos, val = _check(pos, val)
    out = np.empty((q.shape[0], val.shape[1]), np.float64)
    lib.lo_exact_gt_f64(pos.shape[1], val.shape[1], q.shape[0], q, pos.shape[0], pos, val, out)
    return out


def reference_lattice(pos: np.ndarray, val: np.ndarray,
                      slice_pos: np.ndarray | None = None) -> LatticeDump:
    """Drive the reference PermutohedralLattice itself (oracle/_ref)."""
    lib = _load_ref()
    pos, val = _check(pos, val)
    n, d = pos.shape
    vd = val.shape[1]
    h = lib.refh_lattice_create(d, vd, n)
    try:
        lib.refh_lattice_splat(h, pos, val, n)
        m = lib.refh_lattice_size(h)
        keys = np.empty((m, d), np.int16)
        lib.refh_lattice_keys(h, keys)
        rv = np.empty((n, d + 1), np.int32)
        rw = np.empty((n, d + 1), np.float32)
        lib.refh_lattice_replay(h, rv, rw)
        sp = np.empty((m, vd), np.float32)
        lib.refh_lattice_values(h, sp)
        lib.refh_lattice_blur(h)
        bl = np.empty((m, vd), np.float32)
        lib.refh_lattice_values(h, bl)
        if slice_pos is None:
            out = np.empty((n, vd), np.float32)
            lib.refh_lattice_slice_replay(h, out, n)
        else:
            sp_ = np.ascontiguousarray(slice_pos, dtype=np.float32)
            out = np.empty((sp_.shape[0], vd), np.float32)
            lib.refh_lattice_slice_positions(h, sp_, out, sp_.shape[0])
        return LatticeDump(keys, rv, rw, sp, bl, out)
    finally:
        lib.refh_lattice_destroy(h)


def reference_bilateral(img: np.ndarray, sigma_s: float, sigma_r: float,
                        sigma_t: float = 0.0, sigma_s_y: float | None = None,
                        method: str = "permutohedral") -> tuple[np.ndarray, float]:
    """Bilateral::apply on a planar (c, h, w) or (c, f, h, w) image; returns (out, seconds)."""
    lib = _load_ref()
    a = np.ascontiguousarray(img, dtype=np.float32).copy()
    if a.ndim == 3:
        c, h, w = a.shape
        f = 1
    else:
        c, f, h, w = a.shape
    sy = sigma_s if sigma_s_y is None else sigma_s_y
    t = lib.refh_bilateral(a, w, h, f, c, sigma_s, sy, sigma_t, sigma_r, METHODS[method])
    if t < 0:
        raise RuntimeError(lib.refh_last_error().decode())
    return a, t


def reference_joint_bilateral(img: np.ndarray, ref: np.ndarray, sigma_s: float, sigma_r: float,
                              sigma_t: float = 0.0, sigma_s_y: float | None = None,
                              method: str = "permutohedral") -> tuple[np.ndarray, float]:
    lib = _load_ref()
    a = np.ascontiguousarray(img, dtype=np.float32).copy()
    b = np.ascontiguousarray(ref, dtype=np.float32)
    if a.ndim == 3:
        c, h, w = a.shape
        f = 1
        cr = b.shape[0]
    else:
        c, f, h, w = a.shape
        cr = b.shape[0]
    sy = sigma_s if sigma_s_y is None else sigma_s_y
    t = lib.refh_joint_bilateral(a, b, w, h, f, c, cr, sigma_s, sy, sigma_t, sigma_r,
                                 METHODS[method])
    if t < 0:
        raise RuntimeError(lib.refh_last_error().decode())
    return a, t


def reference_nlmeans3d(vol: np.ndarray, patch: float, dims: int, spatial: float,
                        patch_sigma: float, method: str = "permutohedral"):
    """NLMeans3D::apply on a planar (c, f, h, w) volume (src/GaussTransform.cpp:934-941);
    returns (out, guide, seconds), guide being the (dims, f, h, w) PCA projections the
    joint bilateral filtered against (the reference draws its patches at random)."""
    lib = _load_ref()
    a = np.ascontiguousarray(vol, dtype=np.float32).copy()
    c, f, h, w = a.shape
    guide = np.empty((dims, f, h, w), np.float32)
    t = lib.refh_nlmeans3d(a, guide, w, h, f, c, patch, dims, spatial, patch_sigma,
                           METHODS[method])
    if t < 0:
        raise RuntimeError(lib.refh_last_error().decode())
    return a, guide, t


def reference_gauss_transform(slice_img: np.ndarray | None, splat_img: np.ndarray,
                              values: np.ndarray, sigmas, method: str = "permutohedral"):
    """GaussTransform::apply on planar (c, f, h, w) images; slice_img None = same handle."""
    lib = _load_ref()
    sp = np.ascontiguousarray(splat_img, dtype=np.float32)
    va = np.ascontiguousarray(values, dtype=np.float32)
    if sp.ndim == 3:
        sp = sp[:, None]
        va = va[:, None]
        if slice_img is not None:
            slice_img = slice_img[:, None]
    dpos, f, h, w = sp.shape
    vd = va.shape[0]
    same = 1 if slice_img is None else 0
    sl = sp if slice_img is None else np.ascontiguousarray(slice_img, dtype=np.float32)
    sig = np.ascontiguousarray(np.asarray(sigmas, dtype=np.float32).reshape(-1))
    out = np.empty((vd, f, h, w), np.float32)
    t = lib.refh_gauss_transform(sl, sp, same, va, w, h, f, dpos, vd, sig, METHODS[method], out)
    if t < 0:
        raise RuntimeError(lib.refh_last_error().decode())
    return out, t


def bilateral_points(img: np.ndarray, ref: np.ndarray, sigma_s: float, sigma_r: float,
                     sigma_s_y: float | None = None):
    """Interleaved positions/values exactly as JointBilateral::apply builds them for one
    frame (src/GaussTransform.cpp:646-667): positions (ref*(1/sr)..., x*(1/ss), y*(1/ss)),
    values (img..., 1); both axes filtered."""
    c, h, w = img.shape
    cr = ref.shape[0]
    sy = sigma_s if sigma_s_y is None else sigma_s_y
    inv_r = np.float32(1.0) / np.float32(sigma_r)
    inv_x = np.float32(1.0) / np.float32(sigma_s)
    inv_y = np.float32(1.0) / np.float32(sy)
    pos = np.empty((h, w, cr + 2), np.float32)
    for k in range(cr):
        pos[:, :, k] = ref[k] * inv_r
    pos[:, :, cr] = np.arange(w, dtype=np.float32)[None, :] * inv_x
    pos[:, :, cr + 1] = np.arange(h, dtype=np.float32)[:, None] * inv_y
    val = np.empty((h, w, c + 1), np.float32)
    for k in range(c):
        val[:, :, k] = img[k]
    val[:, :, c] = 1.0
    return pos.reshape(-1, cr + 2), val.reshape(-1, c + 1)


def volume_points(img: np.ndarray, ref: np.ndarray, sigma_s: float, sigma_r: float,
                  sigma_t: float):
    """Positions/values as JointBilateral::apply builds them for a (c, f, h, w) volume
    filtered in x and y (src/GaussTransform.cpp:540-545, 646-667): the points in t, y, x
    loop order, positions (ref*(1/sr)..., x*(1/ss), y*(1/ss)[, t*(1/st)]) where the t
    term is present only when f > 1 and sigma_t < 10 f, values (img..., 1)."""
    c, f, h, w = img.shape
    cr = ref.shape[0]
    filter_t = f > 1 and sigma_t < 10 * f
    dp = cr + 2 + (1 if filter_t else 0)
    inv_r = np.float32(1.0) / np.float32(sigma_r)
    inv_s = np.float32(1.0) / np.float32(sigma_s)
    pos = np.empty((f, h, w, dp), np.float32)
    for k in range(cr):
        pos[..., k] = ref[k] * inv_r
    pos[..., cr] = np.arange(w, dtype=np.float32)[None, None, :] * inv_s
    pos[..., cr + 1] = np.arange(h, dtype=np.float32)[None, :, None] * inv_s
    if filter_t:
        inv_t = np.float32(1.0) / np.float32(sigma_t)
        pos[..., cr + 2] = np.arange(f, dtype=np.float32)[:, None, None] * inv_t
    val = np.empty((f, h, w, c + 1), np.float32)
    for k in range(c):
        val[..., k] = img[k]
    val[..., c] = 1.0
    return pos.reshape(-1, dp), val.reshape(-1, c + 1)
