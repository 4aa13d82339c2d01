"""Several samples of one image per wave (mc_render_params.samples_per_wave):
the accumulation buffer equals one-sample-per-wave rendering bit for bit
(each pixel adds its samples in sample order), for any wave size, with graph
replay or not, persistent or plain trace, with progressive first_sample, and
the ray counts are the same."""
import ctypes as C

import numpy as np
import pytest

import mcpt

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = mcpt.Context(0)
    yield c
    c.close()


_cache = {}


def setup(ctx, kind, variant):
    key = (kind, variant)
    if key not in _cache:
        s = mcpt.generate_scene(kind, variant=variant, seed=2)
        env = mcpt.host_env(s)
        ds = mcpt.DeviceScene(mcpt.host_triangles(s), spheres=mcpt.host_spheres(s), env_rgba=env,
                              env_intensity=s.env_intensity)
        bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4)
        _cache[key] = (s, ds, bvh)
    return _cache[key]


def render(ctx, kind, variant, W, H, spp, spw, first=0, graph=False, persistent=True, depth=8):
    s, ds, bvh = setup(ctx, kind, variant)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = W / float(H)
    mcpt.camera_initialize(cam)
    p = mcpt.render_params(cam, W, H, spp, depth, persistent=persistent, rng=mcpt.RNG_PHILOX, seed=99,
                           first_sample=first, use_graph=graph, samples_per_wave=spw)
    acc = torch.full((W * H * 3,), 0.25, dtype=torch.float32, device="cuda")  # progressive: adds onto what is there
    st = mcpt.RenderStats()
    mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                           C.byref(st)))
    return acc.cpu().numpy(), st


@pytest.mark.parametrize("kind,variant,W,H", [(mcpt.SCENE_CORNELL_BOXES, 0, 96, 80),
                                              (mcpt.SCENE_CORNELL_SPHERES, 0, 64, 64),
                                              (mcpt.SCENE_DISPLACED_ICOSPHERES, 5, 160, 90)])
@pytest.mark.parametrize("spp,spw", [(7, 3), (8, 8), (5, 0), (16, 4)])
def test_samples_per_wave_equal_one_sample_waves(ctx, kind, variant, W, H, spp, spw):
    ref, rs = render(ctx, kind, variant, W, H, spp, 1, first=3)
    got, gs = render(ctx, kind, variant, W, H, spp, spw, first=3)
    assert got.tobytes() == ref.tobytes()
    assert gs.extend_rays == rs.extend_rays and gs.shadow_rays == rs.shadow_rays
    assert gs.paths == rs.paths == W * H * spp


@pytest.mark.parametrize("graph,persistent", [(True, True), (False, False), (True, False)])
def test_samples_per_wave_with_graph_and_plain_trace(ctx, graph, persistent):
    ref, _ = render(ctx, mcpt.SCENE_CORNELL_BOXES, 0, 128, 128, 6, 1, graph=graph, persistent=persistent)
    got, _ = render(ctx, mcpt.SCENE_CORNELL_BOXES, 0, 128, 128, 6, 4, graph=graph, persistent=persistent)
    assert got.tobytes() == ref.tobytes()


def test_samples_per_wave_full_image(ctx):
    """The benchmark's image size: 1920x1080, automatic wave size (4 samples)."""
    ref, rs = render(ctx, mcpt.SCENE_DISPLACED_ICOSPHERES, 6, 1920, 1080, 4, 1)
    got, gs = render(ctx, mcpt.SCENE_DISPLACED_ICOSPHERES, 6, 1920, 1080, 4, 0)
    assert got.tobytes() == ref.tobytes()
    assert gs.extend_rays == rs.extend_rays
