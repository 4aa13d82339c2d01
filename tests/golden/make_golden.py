"""Generates the golden fixtures in tests/golden/ from the UNMODIFIED reference
(oracle/_ref/libmcref*.so: src/path_tracer.cu compiled for sm_100a with the
oracle's compile-only stubs).

  python tests/golden/make_golden.py          # host-side vectors (no GPU needed):
                                              #   Morton codes, std::sort order, bounds,
                                              #   light list, Camera::initialize
  python tests/golden/make_golden.py --gpu    # device-side vectors (B200): reference
                                              #   LBVH nodes, closest/any hits of a ray
                                              #   set, small Philox-mode images

Scenes come from the library's seeded generator (host code); the fixtures hold
the reference's outputs for them. tests/test_cpu.py checks the CPU
oracle against these files; the GPU tests compare the CUDA path against the
reference build directly.
"""
import ctypes as C
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "monocuda-pt_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
import mcpt  # noqa: E402
import mcref  # noqa: E402
from helpers import primary_rays, random_rays  # noqa: E402

SCENES = {"cornell": (mcpt.SCENE_CORNELL_BOXES, 0), "ico3": (mcpt.SCENE_DISPLACED_ICOSPHERES, 3)}


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def host_part(name, kind, variant):
    ref = mcref.load(False)
    s = mcpt.generate_scene(kind, variant=variant, seed=2)
    tris = mcpt.host_triangles(s)
    n = len(tris)
    out = {k: np.zeros(n, np.uint32 if k in ("codes", "sorted") else np.int32) for k in ("codes", "sorted", "ids", "types", "perm")}
    sb = np.zeros(n * 8, np.float32)
    bb = np.zeros(8, np.float32)
    tb = np.zeros(n * 8, np.float32)
    lights = np.zeros(n * 16, np.float32)
    nl = C.c_int32()
    assert ref.mcref_finalize_and_sort(C.addressof(tris), n, None, 0, out["codes"].ctypes.data, out["sorted"].ctypes.data,
                                       out["ids"].ctypes.data, out["types"].ctypes.data, out["perm"].ctypes.data,
                                       sb.ctypes.data, bb.ctypes.data, tb.ctypes.data, lights.ctypes.data, C.byref(nl)) == 0
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    base = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    ref.mcref_camera_initialize(C.addressof(cam))
    tri_bytes = np.frombuffer(tris, dtype=np.uint8).reshape(n, 224)
    data = dict(out, sorted_bounds=sb.reshape(n, 8), scene_bounds=bb,
                lights=lights[: nl.value * 16].reshape(nl.value, 16), camera=np.frombuffer(bytes(cam), np.uint8),
                camera_input=np.frombuffer(bytes(base), np.uint8), scene_sha256=np.array(digest(tri_bytes)))
    mcpt.free_scene(s)
    return data


def full_scene_digests():
    """Digests of the reference's host outputs on the full 3,932,176-triangle scene."""
    ref = mcref.load(False)
    s = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=8, seed=2)
    tris = mcpt.host_triangles(s)
    n = len(tris)
    codes = np.zeros(n, np.uint32)
    srt = np.zeros(n, np.uint32)
    ids = np.zeros(n, np.int32)
    ty = np.zeros(n, np.int32)
    perm = np.zeros(n, np.int32)
    sb = np.zeros(n * 8, np.float32)
    bb = np.zeros(8, np.float32)
    tb = np.zeros(n * 8, np.float32)
    lights = np.zeros(64, np.float32)
    nl = C.c_int32()
    ref.mcref_finalize_and_sort(C.addressof(tris), n, None, 0, codes.ctypes.data, srt.ctypes.data, ids.ctypes.data,
                                ty.ctypes.data, perm.ctypes.data, sb.ctypes.data, bb.ctypes.data, tb.ctypes.data,
                                lights.ctypes.data, C.byref(nl))
    d = {"n": np.array(n), "codes_sha256": np.array(digest(codes)), "sorted_sha256": np.array(digest(srt)),
         "perm_sha256": np.array(digest(perm)), "scene_bounds": bb,
         "scene_sha256": np.array(digest(np.frombuffer(tris, dtype=np.uint8)))}
    mcpt.free_scene(s)
    return d


def gpu_part(name, kind, variant):
    ref = mcref.load(False)
    s = mcpt.generate_scene(kind, variant=variant, seed=2)
    tris = mcpt.host_triangles(s)
    n = len(tris)
    h = np.load(os.path.join(HERE, "%s_host.npz" % name))
    # every NpzFile lookup makes a fresh array: hold them while the reference reads them
    srt = np.ascontiguousarray(h["sorted"], dtype=np.uint32)
    ids = np.ascontiguousarray(h["ids"], dtype=np.int32)
    types = np.ascontiguousarray(h["types"], dtype=np.int32)
    sbounds = np.ascontiguousarray(h["sorted_bounds"], dtype=np.float32)
    assert len(srt) == n and np.all(srt[1:] >= srt[:-1]), "fixture does not match the scene"
    internal = (mcpt.BvhNode * (n - 1))()
    leaves = (mcpt.BvhNode * n)()
    assert ref.mcref_build_bvh(srt.ctypes.data, ids.ctypes.data, types.ctypes.data, sbounds.ctypes.data, n,
                               C.addressof(internal), C.addressof(leaves)) == 0
    env = mcpt.host_env(s)
    assert ref.mcref_scene_upload(C.addressof(tris), n, None, 0, env.ctypes.data if env is not None else None,
                                  s.env_width, s.env_height, s.env_intensity, 0.0) == 0
    if kind == mcpt.SCENE_CORNELL_BOXES:
        rays = np.concatenate([primary_rays(s.camera, s.width, s.height, stride=16),
                               random_rays(3072, (-1.9, 0.1, -3.9), (1.9, 3.9, -0.1), seed=5)], axis=1)
    else:
        rays = np.concatenate([primary_rays(s.camera, s.width, s.height, stride=48),
                               random_rays(3072, -1.5, 1.5, seed=5)], axis=1)
    rays = np.ascontiguousarray(rays)
    nr = rays.shape[1]
    hits = np.zeros((nr, 4), np.int32)
    assert ref.mcref_trace(rays.ctypes.data, nr, 0, None, hits.ctypes.data, None) == 0
    tmax = np.random.default_rng(9).uniform(0.01, 6.0, nr).astype(np.float32)
    occ = np.zeros(nr, np.int32)
    assert ref.mcref_trace(rays.ctypes.data, nr, 2, tmax.ctypes.data, None, occ.ctypes.data) == 0
    refp = mcref.load(True)
    assert refp.mcref_scene_upload(C.addressof(tris), n, None, 0, env.ctypes.data if env is not None else None,
                                   s.env_width, s.env_height, s.env_intensity, 0.0) == 0
    W, H, spp = 64, 48, 8
    img = np.zeros(W * H * 3, np.float32)
    stats = np.zeros(3, np.float64)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    assert refp.mcref_render(C.addressof(cam), W, H, spp, 8, 2, 1234, 0, 0, img.ctypes.data, stats.ctypes.data) == 0
    raw_i = np.frombuffer(bytes(internal), np.uint8).reshape(n - 1, 64)
    raw_l = np.frombuffer(bytes(leaves), np.uint8).reshape(n, 64)
    return {"internal": raw_i, "leaves": raw_l, "rays": rays, "hits": hits, "tmax": tmax, "occluded": occ,
            "image": img.reshape(H, W, 3), "image_spp": np.array(spp), "image_rays": stats[:2]}


def main():
    out_dir = HERE
    if "--out" in sys.argv:
        out_dir = sys.argv[sys.argv.index("--out") + 1]
        os.makedirs(out_dir, exist_ok=True)
    if "--gpu" in sys.argv:
        for name, (kind, variant) in SCENES.items():
            d = gpu_part(name, kind, variant)
            np.savez_compressed(os.path.join(out_dir, "%s_device.npz" % name), **d)
            print("wrote", name, "device fixtures")
        return
    for name, (kind, variant) in SCENES.items():
        d = host_part(name, kind, variant)
        np.savez_compressed(os.path.join(HERE, "%s_host.npz" % name), **d)
        print("wrote", name, "host fixtures", len(d["codes"]), "primitives")
    np.savez_compressed(os.path.join(HERE, "full_icospheres_host_digest.npz"), **full_scene_digests())
    print("wrote full-scene digests")


if __name__ == "__main__":
    main()
