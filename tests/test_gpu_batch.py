"""Batched multi-scene rendering and CUDA-graph replay.

A batch BVH (one build over many scenes) and a batched render (shared waves of
paths from every scene) must produce, for every scene, exactly the image a
single-scene build and render of that scene produces; graph replay must equal
stream launches.
"""
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


def member(i, target):
    s = mcpt.generate_scene(mcpt.SCENE_BATCH_MEMBER, variant=i, seed=3, triangle_target=target)
    return s


def small_params(s, W, spp, first=0):
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = 1.0
    mcpt.camera_initialize(cam)
    return mcpt.render_params(cam, W, W, spp, 8, persistent=True, rng=mcpt.RNG_PHILOX, seed=99, first_sample=first)


def test_batch_matches_single_scene_renders(ctx):
    specs = [(0, 3000, 64, 3), (1, 5000, 96, 2), (2, 2000, 48, 4), (3, 8000, 80, 1), (4, 4000, 64, 2), (5, 3000, 32, 3)]
    scenes = [member(i, t) for i, t, _, _ in specs]
    devs = [mcpt.DeviceScene(mcpt.host_triangles(s)) for s in scenes]
    batch = mcpt.BatchBvh(ctx, [d.view for d in devs], layout=mcpt.LAYOUT_WIDE4)
    accs = [torch.zeros(W * W * 3, dtype=torch.float32, device="cuda") for _, _, W, _ in specs]
    items = []
    for (i, t, W, spp), d, a, s in zip(specs, devs, accs, scenes):
        items.append(mcpt.BatchItem(d.view, small_params(s, W, spp), a.data_ptr()))
    st = batch.render(items)
    assert st.paths == sum(W * W * spp for _, _, W, spp in specs)
    for k, ((i, t, W, spp), d, a, s) in enumerate(zip(specs, devs, accs, scenes)):
        single = mcpt.Bvh(ctx, d.view, layout=mcpt.LAYOUT_WIDE4)
        ref = torch.zeros_like(a)
        p = small_params(s, W, spp)
        rs = mcpt.RenderStats()
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, single.handle, C.byref(d.view), C.byref(p), ref.data_ptr(),
                                               C.byref(rs)))
        assert torch.equal(a, ref), "scene %d differs from its single-scene render" % k
        assert float(a.sum()) > 0
    for s in scenes:
        mcpt.free_scene(s)


def test_batch_graph_replay_equals_stream_launches(ctx):
    specs = [(7, 3000, 64, 3), (8, 6000, 48, 2), (9, 2500, 72, 4)]
    scenes = [member(i, t) for i, t, _, _ in specs]
    devs = [mcpt.DeviceScene(mcpt.host_triangles(s)) for s in scenes]
    batch = mcpt.BatchBvh(ctx, [d.view for d in devs], layout=mcpt.LAYOUT_WIDE4)
    outs = []
    for graph in (False, True, True):
        accs = [torch.zeros(W * W * 3, dtype=torch.float32, device="cuda") for _, _, W, _ in specs]
        items = [mcpt.BatchItem(d.view, small_params(s, W, spp), a.data_ptr())
                 for (_, _, W, spp), d, a, s in zip(specs, devs, accs, scenes)]
        st = batch.render(items, use_graph=graph)
        outs.append((torch.cat(accs).cpu().numpy(), st.extend_rays, st.shadow_rays))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[1][0], outs[2][0])
    assert outs[0][1:] == outs[1][1:] == outs[2][1:]
    for s in scenes:
        mcpt.free_scene(s)


def test_single_scene_graph_mode_identical(ctx):
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_SPHERES)
    d = mcpt.DeviceScene(mcpt.host_triangles(s), spheres=mcpt.host_spheres(s))
    b = mcpt.Bvh(ctx, d.view, layout=mcpt.LAYOUT_WIDE4)
    res = []
    for graph in (False, True):
        acc = torch.zeros(128 * 128 * 3, dtype=torch.float32, device="cuda")
        p = small_params(s, 128, 4)
        p.use_graph = 1 if graph else 0
        st = mcpt.RenderStats()
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, b.handle, C.byref(d.view), C.byref(p), acc.data_ptr(),
                                               C.byref(st)))
        res.append(acc.cpu().numpy())
    assert np.array_equal(res[0], res[1])
    mcpt.free_scene(s)


def test_batch_rejects_mismatched_items(ctx):
    scenes = [member(i, 2000) for i in (10, 11)]
    devs = [mcpt.DeviceScene(mcpt.host_triangles(s)) for s in scenes]
    batch = mcpt.BatchBvh(ctx, [d.view for d in devs])
    acc = torch.zeros(32 * 32 * 3, dtype=torch.float32, device="cuda")
    one = [mcpt.BatchItem(devs[0].view, small_params(scenes[0], 32, 1), acc.data_ptr())]
    with pytest.raises(mcpt.McError):
        batch.render(one)  # 1 item for a 2-scene build
    swapped = [mcpt.BatchItem(devs[1].view, small_params(scenes[1], 32, 1), acc.data_ptr()),
               mcpt.BatchItem(devs[0].view, small_params(scenes[0], 32, 1), acc.data_ptr())]
    if devs[0].n != devs[1].n:
        with pytest.raises(mcpt.McError):
            batch.render(swapped)
    for s in scenes:
        mcpt.free_scene(s)


def test_autotune_returns_params_that_leave_the_image_unchanged(ctx):
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_SPHERES)
    d = mcpt.DeviceScene(mcpt.host_triangles(s), spheres=mcpt.host_spheres(s))
    b = mcpt.Bvh(ctx, d.view, layout=mcpt.LAYOUT_WIDE4)
    p = small_params(s, 96, 4)
    tuned = mcpt.RenderParams.from_buffer_copy(bytes(p))
    mcpt.check(ctx.lib.mc_autotune(ctx.handle, b.handle, C.byref(d.view), C.byref(tuned), 3000))
    assert tuned.persistent in (0, 1) and 1 <= tuned.refill_threshold <= 32 and tuned.use_graph in (0, 1)
    again = mcpt.RenderParams.from_buffer_copy(bytes(p))
    mcpt.check(ctx.lib.mc_autotune(ctx.handle, b.handle, C.byref(d.view), C.byref(again), 3000))  # cached
    assert (again.persistent, again.refill_threshold, again.use_graph) == \
        (tuned.persistent, tuned.refill_threshold, tuned.use_graph)
    imgs = []
    for q in (p, tuned):
        acc = torch.zeros(96 * 96 * 3, dtype=torch.float32, device="cuda")
        st = mcpt.RenderStats()
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, b.handle, C.byref(d.view), C.byref(q), acc.data_ptr(),
                                               C.byref(st)))
        imgs.append(acc.cpu().numpy())
    assert np.array_equal(imgs[0], imgs[1])
    mcpt.free_scene(s)
