"""Shared helpers for the tests: scene upload, ray sets, oracle calls."""
import ctypes as C
import os

import numpy as np

import mcpt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")

_orc = None


def oracle():
    """The CPU restatement (oracle/liboracle.so)."""
    global _orc
    if _orc is None:
        lib = C.CDLL(ORACLE_LIB)
        P, I = C.c_void_p, C.c_int
        lib.orc_finalize_sort.argtypes = [P, I, P, I, P, P, P, P, P]
        lib.orc_build.argtypes = [P, P, P, I, I, P, P]
        lib.orc_depth.argtypes = [P, P, I]
        lib.orc_trace.argtypes = [P, P, P, I, P, P, P, I, I, P, P, P, I]
        lib.orc_scene_create.restype = P
        lib.orc_scene_create.argtypes = [P, I, P, I, P, I, I, C.c_float, C.c_float]
        lib.orc_scene_destroy.argtypes = [P]
        lib.orc_render.argtypes = [P, P, I, I, I, I, I, C.c_uint64, I, I, I, I, I, I, I, P, P]
        lib.orc_philox4x32_10.argtypes = [P, P, P]
        lib.orc_guide_forward.argtypes = [P, P, I, P, P, I, P]
        lib.orc_guide_loss_grad.argtypes = [P, P, I, P, P, I, P, P]
        _orc = lib
    return _orc


def tri_bytes(tris):
    return np.frombuffer(tris, dtype=np.uint8).reshape(len(tris), 224)


def oracle_sort(tris):
    n = len(tris)
    codes = np.zeros(n, np.uint32)
    srt = np.zeros(n, np.uint32)
    perm = np.zeros(n, np.int32)
    boxes = np.zeros(n * 8, np.float32)
    sb = np.zeros(8, np.float32)
    oracle().orc_finalize_sort(C.addressof(tris), n, None, 0, codes.ctypes.data, srt.ctypes.data, perm.ctypes.data,
                               boxes.ctypes.data, sb.ctypes.data)
    return codes, srt, perm, boxes.reshape(n, 8), sb


def oracle_build(srt, perm, boxes, ns=0):
    n = len(srt)
    internal = (mcpt.BvhNode * max(n - 1, 1))()
    leaves = (mcpt.BvhNode * n)()
    oracle().orc_build(srt.ctypes.data, perm.ctypes.data, boxes.ctypes.data, n, ns, C.addressof(internal),
                       C.addressof(leaves))
    return internal, leaves


def node_fields(nodes, count):
    """(bounds float32 [count, 8], left, right, lleaf, rleaf, parent, prim, isleaf) from BvhNode arrays."""
    raw = np.frombuffer(nodes, dtype=np.uint8, count=count * 64).reshape(count, 64)
    bounds = raw[:, 0:32].copy().view(np.float32)
    ints = raw[:, 32:56].copy()
    left = ints[:, 0:4].copy().view(np.int32).ravel()
    right = ints[:, 4:8].copy().view(np.int32).ravel()
    lleaf = raw[:, 40].copy()
    rleaf = raw[:, 41].copy()
    parent = raw[:, 44:48].copy().view(np.int32).ravel()
    prim = raw[:, 48:52].copy().view(np.int32).ravel()
    isleaf = raw[:, 52].copy()
    return bounds, left, right, lleaf, rleaf, parent, prim, isleaf


def primary_rays(cam, W, H, stride=1):
    """Pixel-centre camera rays (Camera::getRay with aperture 0, PT:1648-1658) as SoA float32 [7, n]."""
    xs, ys = np.meshgrid(np.arange(0, W, stride), np.arange(0, H, stride))
    xs = xs.ravel().astype(np.float32)
    ys = ys.ravel().astype(np.float32)
    p00 = np.array([cam.pixel00.x, cam.pixel00.y, cam.pixel00.z], np.float32)
    du = np.array([cam.pixel_delta_u.x, cam.pixel_delta_u.y, cam.pixel_delta_u.z], np.float32)
    dv = np.array([cam.pixel_delta_v.x, cam.pixel_delta_v.y, cam.pixel_delta_v.z], np.float32)
    c = np.array([cam.center.x, cam.center.y, cam.center.z], np.float32)
    pc = p00[None, :] + du[None, :] * xs[:, None] + dv[None, :] * ys[:, None]
    d = pc - c[None, :]
    d = d / np.sqrt((d * d).sum(1, keepdims=True))
    n = len(xs)
    r = np.zeros((7, n), np.float32)
    r[0:3] = c[:, None]
    r[3:6] = d.T
    r[6] = 0.5
    return np.ascontiguousarray(r)


def random_rays(n, lo, hi, seed):
    """Origins uniform in the box [lo, hi], directions uniform on the sphere."""
    g = np.random.default_rng(seed)
    o = g.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = g.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((7, n), np.float32)
    r[0:3] = o.T
    r[3:6] = d.T
    r[6] = g.uniform(0, 1, n).astype(np.float32)
    return np.ascontiguousarray(r)


def ulp_diff(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)
