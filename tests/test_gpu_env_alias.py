"""Alias-table environment sampling (MC_ENV_SAMPLE_ALIAS) against the
reference's CDF inversion (PT:433-467) and the FP64 host oracle.

The alias table draws texels from the same distribution as the CDFs but is not
draw-compatible with them, so the check is statistical: on the displaced
icospheres scene with the benchmark's 2048x1024 procedural sky (a 2-degree sun
of radiance ~600 that next-event estimation must find), independent batches
of the alias-mode image agree with the CDF-mode image and with the FP64
oracle (which samples by CDF inversion) in expectation: colour-channel means
within 3 standard errors, 4x4 tiles within 4. Both GPU modes keep the firefly
clamp, as the oracle does.
"""
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
def sky_scene():
    ctx = mcpt.Context(0)
    s = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=3, seed=2)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = 1.0
    mcpt.camera_initialize(cam)
    tris = mcpt.host_triangles(s)
    env = mcpt.host_env(s)
    ds = mcpt.DeviceScene(tris, env_rgba=env, env_intensity=s.env_intensity)
    bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4)
    yield ctx, s, cam, tris, env, ds, bvh
    bvh.close()
    ds.close()
    ctx.close()


def gpu_batches(ctx, ds, bvh, cam, depth, mode, seed):
    out = []
    for b in range(BATCHES):
        acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        p = mcpt.render_params(cam, W, H, SPP, depth, rng=mcpt.RNG_PHILOX, seed=seed, first_sample=b * SPP,
                               env_sampling=mode)
        st = mcpt.RenderStats()
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               C.byref(st)))
        out.append(acc.cpu().numpy().astype(np.float64).reshape(H, W, 3) / SPP)
    return np.array(out)


def tiles(img):
    return img.reshape(4, H // 4, 4, W // 4, 3).mean(axis=(1, 3)).reshape(16, 3)


def agree(a, b, k, rel=0.0):
    """Means within k standard errors, plus `rel` of the mean: a tile that
    sees only the sky has no variance, and the oracle's restatement of the
    texture unit's bilinear filtering agrees with it to about 1e-4, not bit
    for bit."""
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
    diff = np.abs(a.mean(0) - b.mean(0))
    tol = k * se + rel * np.abs(b.mean(0)) + 1e-7
    return diff / np.maximum(se, 1e-12), bool(np.all(diff <= tol))


def test_alias_sampling_converges_to_cdf_sampling_and_the_fp64_oracle(sky_scene):
    ctx, s, cam, tris, env, ds, bvh = sky_scene
    alias = gpu_batches(ctx, ds, bvh, cam, s.max_depth, mcpt.ENV_SAMPLE_ALIAS, 777)
    cdf = gpu_batches(ctx, ds, bvh, cam, s.max_depth, mcpt.ENV_SAMPLE_CDF, 1234)
    orc = oracle()
    h = orc.orc_scene_create(C.addressof(tris), len(tris), None, 0, env.ctypes.data, s.env_width, s.env_height,
                             s.env_intensity, 0.0)
    ref = []
    for b in range(BATCHES):
        acc = np.zeros(W * H * 3, np.float64)
        orc.orc_render(h, C.addressof(cam), W, H, SPP, b * SPP, s.max_depth, 987654321, 1, 0, 0, 0, W, H,
                       os.cpu_count() or 1, acc.ctypes.data, None)
        ref.append(acc.reshape(H, W, 3) / SPP)
    orc.orc_scene_destroy(h)
    ref = np.array(ref)
    for name, other, rel in (("cdf", cdf, 0.0), ("fp64 oracle", ref, 1e-3)):
        z, ok = agree(alias.mean(axis=(1, 2)), other.mean(axis=(1, 2)), 3.0, rel)
        print("alias vs %s: means %s vs %s, diff/se %s" % (name, alias.mean(axis=(0, 1, 2)),
                                                          other.mean(axis=(0, 1, 2)), z))
        assert ok, name
        tz, tok = agree(np.array([tiles(g) for g in alias]), np.array([tiles(r) for r in other]), 4.0, rel)
        print("  worst tile diff/se %.2f" % float(tz.max()))
        assert tok, name
    # the sky carries light into the image: a render without it is darker
    assert alias.mean() > 0.05


def test_alias_sampling_is_deterministic_and_differs_from_cdf_draws(sky_scene):
    ctx, s, cam, tris, env, ds, bvh = sky_scene
    imgs = []
    for mode in (mcpt.ENV_SAMPLE_ALIAS, mcpt.ENV_SAMPLE_ALIAS, mcpt.ENV_SAMPLE_CDF):
        acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        p = mcpt.render_params(cam, W, H, 4, s.max_depth, rng=mcpt.RNG_PHILOX, seed=5, env_sampling=mode)
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               None))
        imgs.append(acc.cpu().numpy())
    assert np.array_equal(imgs[0], imgs[1])
    assert not np.array_equal(imgs[0], imgs[2])


def test_alias_sampling_needs_a_library_made_map(sky_scene):
    """A map whose tables the library did not build has no alias table: the
    render is refused instead of sampling from memory that is not one."""
    ctx, s, cam, tris, env, ds, bvh = sky_scene
    foreign = torch.zeros(s.env_height * (s.env_width + 1), dtype=torch.float32, device="cuda")
    view = mcpt.SceneView.from_buffer_copy(bytes(ds.view))
    view.env.col_cdf = foreign.data_ptr()
    acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    p = mcpt.render_params(cam, W, H, 1, s.max_depth, rng=mcpt.RNG_PHILOX, seed=5, env_sampling=mcpt.ENV_SAMPLE_ALIAS)
    assert ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(view), C.byref(p), acc.data_ptr(), None) == 1
    assert b"alias" in ctx.lib.mc_last_error()
    p.env_sampling = 7
    assert ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(), None) == 1
