"""Converged radiance against the FP64 host oracle (oracle/mc_oracle.cpp with
use_double, the reference's integrator in double precision): with independent
seeds, the GPU image and the oracle's agree in expectation. Per colour
channel the image means differ by less than 3 standard errors, and on a 4x4
grid of tiles by less than 4 (48 comparisons per scene). Both estimators keep
the reference's firefly clamp, so they estimate the same quantity."""
import ctypes as C
import os

import numpy as np
import pytest

import mcpt
from helpers import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

W = H = 32
BATCHES, SPP = 8, 64


@pytest.fixture(scope="module")
def ctx():
    c = mcpt.Context(0)
    yield c
    c.close()


def _tiles(img):
    return img.reshape(4, H // 4, 4, W // 4, 3).mean(axis=(1, 3)).reshape(16, 3)


@pytest.mark.parametrize("kind", [mcpt.SCENE_CORNELL_BOXES, mcpt.SCENE_CORNELL_SPHERES])
def test_gpu_image_converges_to_the_fp64_oracle(ctx, kind):
    s = mcpt.generate_scene(kind)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = 1.0
    mcpt.camera_initialize(cam)
    tris = mcpt.host_triangles(s)
    sph = mcpt.host_spheres(s)
    ds = mcpt.DeviceScene(tris, spheres=sph)
    bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4)
    gpu = []
    for b in range(BATCHES):
        acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        p = mcpt.render_params(cam, W, H, SPP, s.max_depth, rng=mcpt.RNG_PHILOX, seed=1234, first_sample=b * SPP)
        st = mcpt.RenderStats()
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               C.byref(st)))
        gpu.append(acc.cpu().numpy().astype(np.float64).reshape(H, W, 3) / SPP)
    bvh.close()
    orc = oracle()
    h = orc.orc_scene_create(C.addressof(tris), len(tris), C.addressof(sph) if sph is not None else None,
                             s.sphere_count, None, 0, 0, 1.0, 0.0)
    ref = []
    for b in range(BATCHES):
        acc = np.zeros(W * H * 3, np.float64)
        orc.orc_render(h, C.addressof(cam), W, H, SPP, b * SPP, s.max_depth, 987654321, 1, 0, 0, 0, W, H,
                       os.cpu_count() or 1, acc.ctypes.data, None)
        ref.append(acc.reshape(H, W, 3) / SPP)
    orc.orc_scene_destroy(h)
    gpu, ref = np.array(gpu), np.array(ref)

    def check(a, b, k):
        se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
        diff = np.abs(a.mean(0) - b.mean(0))
        return diff, se, np.all(diff <= k * se + 1e-7)

    diff, se, ok = check(gpu.mean(axis=(1, 2)), ref.mean(axis=(1, 2)), 3.0)
    print("scene %d: means %s vs %s, diff/se %s" % (kind, gpu.mean(axis=(0, 1, 2)), ref.mean(axis=(0, 1, 2)),
                                                   diff / np.maximum(se, 1e-12)))
    assert ok
    tdiff, tse, tok = check(np.array([_tiles(g) for g in gpu]), np.array([_tiles(r) for r in ref]), 4.0)
    print("  worst tile diff/se %.2f" % float((tdiff / np.maximum(tse, 1e-12)).max()))
    assert tok
    mcpt.free_scene(s)
