"""The wide layouts' binary tree (mc_bvh_build_opts.builder): the clustered
tree (PLOC over the Morton-sorted leaves) and the reference's LBVH give the
same closest hits to the bit (t and primitive), the same any-hit answers and
the same images, because leaves keep the reference's rank for ties; the
clustered tree needs fewer node visits."""
import ctypes as C

import numpy as np
import pytest

import mcpt
from helpers import random_rays

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = mcpt.Context(0)
    yield c
    c.close()


CASES = [(mcpt.SCENE_CORNELL_BOXES, 0), (mcpt.SCENE_DISPLACED_ICOSPHERES, 5), (mcpt.SCENE_CORNELL_SPHERES, 0)]


def _scene(kind, variant):
    s = mcpt.generate_scene(kind, variant=variant, seed=2)
    ds = mcpt.DeviceScene(mcpt.host_triangles(s), spheres=mcpt.host_spheres(s))
    return s, ds


@pytest.mark.parametrize("layout", [mcpt.LAYOUT_WIDE4, mcpt.LAYOUT_WIDE4Q])
@pytest.mark.parametrize("kind,variant", CASES)
def test_clustered_tree_gives_the_same_hits(ctx, kind, variant, layout):
    s, ds = _scene(kind, variant)
    v = np.frombuffer(mcpt.host_triangles(s), np.uint8).reshape(-1, 224)[:, :36].copy().view(np.float32).reshape(-1, 3)
    rays = random_rays(200000, v.min(0), v.max(0), seed=variant + 11)
    out = {}
    for b in (mcpt.BUILDER_LBVH, mcpt.BUILDER_CLUSTERED):
        bvh = mcpt.Bvh(ctx, ds.view, layout=layout, builder=b)
        d_rays = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
        hits = torch.zeros(rays.shape[1] * 4, dtype=torch.int32, device="cuda")
        mcpt.check(ctx.lib.mc_trace_closest(ctx.handle, bvh.handle, C.byref(ds.view), d_rays.data_ptr(), rays.shape[1], 0,
                                            hits.data_ptr()))
        occ = torch.zeros(rays.shape[1], dtype=torch.int32, device="cuda")
        tmax = torch.full((rays.shape[1],), 2.0, dtype=torch.float32, device="cuda")
        mcpt.check(ctx.lib.mc_trace_any(ctx.handle, bvh.handle, C.byref(ds.view), d_rays.data_ptr(), tmax.data_ptr(),
                                        rays.shape[1], 0, occ.data_ptr()))
        out[b] = (hits.cpu().numpy(), occ.cpu().numpy())
        bvh.close()
    assert np.array_equal(out[mcpt.BUILDER_LBVH][0], out[mcpt.BUILDER_CLUSTERED][0])
    assert np.array_equal(out[mcpt.BUILDER_LBVH][1], out[mcpt.BUILDER_CLUSTERED][1])
    mcpt.free_scene(s)


def test_clustered_tree_same_image_fewer_visits(ctx):
    s, ds = _scene(mcpt.SCENE_DISPLACED_ICOSPHERES, 6)
    W, H = 320, 180
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = W / H
    mcpt.camera_initialize(cam)
    res = {}
    for b in (mcpt.BUILDER_LBVH, mcpt.BUILDER_CLUSTERED):
        bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4, builder=b)
        acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        p = mcpt.render_params(cam, W, H, 4, 8, instrument=1)
        st = mcpt.RenderStats()
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               C.byref(st)))
        res[b] = (acc.cpu().numpy(), st.node_visits, st.extend_rays + st.shadow_rays)
        bvh.close()
    assert res[mcpt.BUILDER_LBVH][0].tobytes() == res[mcpt.BUILDER_CLUSTERED][0].tobytes()
    assert res[mcpt.BUILDER_LBVH][2] == res[mcpt.BUILDER_CLUSTERED][2]
    assert res[mcpt.BUILDER_CLUSTERED][1] < 0.8 * res[mcpt.BUILDER_LBVH][1], (res[1][1], res[0][1])
    mcpt.free_scene(s)


def test_batch_build_uses_clustered_trees_per_scene(ctx):
    scenes = [_scene(mcpt.SCENE_BATCH_MEMBER, v) for v in (1, 2, 3)]
    views = [d.view for _, d in scenes]
    hits = {}
    for b in (mcpt.BUILDER_LBVH, mcpt.BUILDER_CLUSTERED):
        bb = mcpt.BatchBvh(ctx, views, layout=mcpt.LAYOUT_WIDE4, builder=b)
        items = []
        accs = []
        for s, d in scenes:
            cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
            cam.image_width = 64
            cam.aspect_ratio = 1.0
            mcpt.camera_initialize(cam)
            acc = torch.zeros(64 * 64 * 3, dtype=torch.float32, device="cuda")
            accs.append(acc)
            it = mcpt.BatchItem()
            it.scene = d.view
            it.params = mcpt.render_params(cam, 64, 64, 3, 8)
            it.d_accum = acc.data_ptr()
            items.append(it)
        bb.render(items)
        torch.cuda.synchronize()
        hits[b] = [a.cpu().numpy().tobytes() for a in accs]
        bb.close()
    assert hits[mcpt.BUILDER_LBVH] == hits[mcpt.BUILDER_CLUSTERED]
    for s, _ in scenes:
        mcpt.free_scene(s)


def _tiny_scene(n_tris, seed):
    """n_tris random triangles with the default material, as a DeviceScene."""
    rng = np.random.default_rng(seed)
    arr = (mcpt.Triangle * n_tris)()
    for i in range(n_tris):
        c = rng.uniform(-1, 1, 3)
        for k, name in enumerate(("v0", "v1", "v2")):
            p = c + rng.uniform(-0.3, 0.3, 3)
            setattr(arr[i], name, mcpt.Vec3(*p.astype(np.float32)))
    return arr, mcpt.DeviceScene(arr)


@pytest.mark.parametrize("n_tris", [1, 2, 3, 17])
def test_tiny_scenes_build_and_agree(ctx, n_tris):
    """One primitive has no tree to cluster (the build keeps the LBVH's
    collapse); two or more cluster. Either way the hits equal the LBVH's."""
    tris, ds = _tiny_scene(n_tris, seed=n_tris)
    rays = random_rays(5000, np.full(3, -1.5), np.full(3, 1.5), seed=3)
    out = []
    for b in (mcpt.BUILDER_LBVH, mcpt.BUILDER_CLUSTERED):
        bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4, builder=b)
        d_rays = torch.from_numpy(rays).cuda()
        hits = torch.zeros(rays.shape[1] * 4, dtype=torch.int32, device="cuda")
        mcpt.check(ctx.lib.mc_trace_closest(ctx.handle, bvh.handle, C.byref(ds.view), d_rays.data_ptr(), rays.shape[1], 0,
                                            hits.data_ptr()))
        out.append(hits.cpu().numpy())
        bvh.close()
    assert np.array_equal(out[0], out[1])
    assert (out[0].reshape(-1, 4)[:, 3] == 1).any()


def test_batch_with_the_smallest_scenes(ctx):
    """A batch whose smallest scene has two primitives clusters it like the
    others and gives the images of the LBVH build. A one-primitive scene in a
    batch is rejected with MC_ERR_INVALID by either builder."""
    small = _tiny_scene(2, seed=5)
    big = _scene(mcpt.SCENE_BATCH_MEMBER, 4)
    views = [small[1].view, big[1].view]
    imgs = {}
    for b in (mcpt.BUILDER_LBVH, mcpt.BUILDER_CLUSTERED):
        bb = mcpt.BatchBvh(ctx, views, layout=mcpt.LAYOUT_WIDE4, builder=b)
        cam = mcpt.Camera.from_buffer_copy(bytes(big[0].camera))
        cam.image_width = 48
        cam.aspect_ratio = 1.0
        mcpt.camera_initialize(cam)
        accs, items = [], []
        for v in views:
            acc = torch.zeros(48 * 48 * 3, dtype=torch.float32, device="cuda")
            it = mcpt.BatchItem()
            it.scene = v
            it.params = mcpt.render_params(cam, 48, 48, 2, 8)
            it.d_accum = acc.data_ptr()
            accs.append(acc)
            items.append(it)
        bb.render(items)
        torch.cuda.synchronize()
        imgs[b] = [a.cpu().numpy().tobytes() for a in accs]
        bb.close()
    assert imgs[mcpt.BUILDER_LBVH] == imgs[mcpt.BUILDER_CLUSTERED]
    one = _tiny_scene(1, seed=6)
    for b in (mcpt.BUILDER_LBVH, mcpt.BUILDER_CLUSTERED):
        with pytest.raises(mcpt.McError) as e:
            mcpt.BatchBvh(ctx, [one[1].view, big[1].view], layout=mcpt.LAYOUT_WIDE4, builder=b)
        assert e.value.status == 1  # MC_ERR_INVALID
    mcpt.free_scene(big[0])


PERSISTENT_CASES = [(mcpt.SCENE_CORNELL_BOXES, 0, mcpt.LAYOUT_WIDE4), (mcpt.SCENE_CORNELL_SPHERES, 0, mcpt.LAYOUT_WIDE4),
                    (mcpt.SCENE_DISPLACED_ICOSPHERES, 7, mcpt.LAYOUT_WIDE4),
                    (mcpt.SCENE_DISPLACED_ICOSPHERES, 5, mcpt.LAYOUT_WIDE4Q),
                    (mcpt.SCENE_DISPLACED_ICOSPHERES, 5, mcpt.LAYOUT_WIDE4)]


@pytest.mark.parametrize("kind,variant,layout", PERSISTENT_CASES)
@pytest.mark.parametrize("builder", [mcpt.BUILDER_CLUSTERED, mcpt.BUILDER_LBVH])
def test_persistent_build_loops_give_the_same_tree(ctx, kind, variant, layout, builder):
    """The clustering rounds and the collapse levels as one cooperative launch
    each build, byte for byte, the tree of the launch-per-phase loops: the same
    node array, the same leaf-ordered primitives, the same level count."""
    s, ds = _scene(kind, variant)
    out = []
    for phase in (False, True):
        bvh = mcpt.Bvh(ctx, ds.view, layout=layout, builder=builder, phase_launches=phase)
        nodes, prims = bvh.traversal_arrays()
        i = bvh.info()
        out.append((nodes.cpu().numpy(), prims.cpu().numpy(), int(i.wide_levels), int(i.node_bytes)))
        bvh.close()
    (n0, p0, l0, b0), (n1, p1, l1, b1) = out
    assert (l0, b0) == (l1, b1)
    assert n0.tobytes() == n1.tobytes()
    assert p0.tobytes() == p1.tobytes()
    mcpt.free_scene(s)


def test_persistent_build_loops_give_the_same_batched_trees(ctx):
    """The same for one batched build over 24 scenes of different sizes."""
    scenes = [mcpt.generate_scene(mcpt.SCENE_BATCH_MEMBER, variant=i, seed=3, triangle_target=2000 + 3000 * i)
              for i in range(24)]
    devs = [mcpt.DeviceScene(mcpt.host_triangles(s)) for s in scenes]
    out = []
    for phase in (False, True):
        b = mcpt.BatchBvh(ctx, [d.view for d in devs], phase_launches=phase)
        nodes, prims = mcpt.traversal_arrays(ctx.lib, b.handle)
        out.append((nodes.cpu().numpy().tobytes(), prims.cpu().numpy().tobytes()))
        b.close()
    assert out[0] == out[1]
    for s in scenes:
        mcpt.free_scene(s)
