"""The render server: shared waves give every request exactly the image a
standalone render of it gives, admission follows the HBM budget in arrival
order, and guided requests complete."""
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


def _scene(i, target):
    s = mcpt.generate_scene(mcpt.SCENE_BATCH_MEMBER, variant=i, seed=3, triangle_target=target)
    return s, mcpt.DeviceScene(mcpt.host_triangles(s))


def _params(s, W, spp, seed=11):
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = 1.0
    mcpt.camera_initialize(cam)
    return mcpt.render_params(cam, W, W, spp, 8, persistent=True, rng=mcpt.RNG_PHILOX, seed=seed)


def _drain(srv, limit=10000):
    for _ in range(limit):
        if srv.step() == 0 and srv.stats().pending == 0:
            return
    raise AssertionError("server did not drain")


def test_shared_waves_equal_standalone_renders(ctx):
    scenes = [_scene(i, t) for i, t in ((20, 3000), (21, 6000), (22, 2000))]
    srv = mcpt.Server(ctx, samples_per_step=2)
    sids = [srv.add_scene(d) for _, d in scenes]
    reqs = [(0, 48, 3), (1, 64, 5), (2, 32, 1), (0, 40, 4), (1, 24, 2)]
    rids = [srv.submit(sids[k], _params(scenes[k][0], W, spp)) for k, W, spp in reqs]
    _drain(srv)
    for rid, (k, W, spp) in zip(rids, reqs):
        r = srv.result(rid)
        assert r.state == mcpt.REQ_DONE and r.spp_done == spp and r.done_s >= r.admit_s >= r.submit_s
        host = srv.read(rid, W, W)
        s, d = scenes[k]
        bvh = mcpt.Bvh(ctx, d.view, layout=mcpt.LAYOUT_WIDE4)
        ref = torch.zeros(W * W * 3, dtype=torch.float32, device="cuda")
        p = _params(s, W, spp)
        st = mcpt.RenderStats()
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(d.view), C.byref(p), ref.data_ptr(),
                                               C.byref(st)))
        assert np.array_equal(host, ref.cpu().numpy()), "request %d differs from its standalone render" % rid
        srv.release(rid)
        bvh.close()
    assert srv.stats().active == 0
    srv.close()
    for s, _ in scenes:
        mcpt.free_scene(s)


def test_admission_follows_the_budget(ctx):
    s, d = _scene(23, 2000)
    probe = mcpt.Server(ctx)
    sid = probe.add_scene(d)
    scene_bytes = probe.stats().scene_bytes
    probe.close()
    W = 64
    # one sample per step: a request's share of the wave buffers is one path per pixel
    per_request = W * W * (12 + 29 * 4 + 1 + 16 + 2)
    # room for the scene and one request at a time
    srv = mcpt.Server(ctx, budget_bytes=scene_bytes + per_request + per_request // 2, samples_per_step=1)
    sid = srv.add_scene(d)
    a = srv.submit(sid, _params(s, W, 3))
    b = srv.submit(sid, _params(s, W, 2))
    srv.step()
    st = srv.stats()
    assert st.active == 1 and st.pending == 1
    while srv.result(a).state != mcpt.REQ_DONE:
        srv.step()
    srv.step()  # b still waits: a's buffer is charged until it is released
    assert srv.result(b).state == mcpt.REQ_PENDING
    srv.release(a)
    _drain(srv)
    rb = srv.result(b)
    assert rb.state == mcpt.REQ_DONE and rb.admit_s >= srv.result(a).done_s
    with pytest.raises(mcpt.McError) as e:
        srv.submit(sid, _params(s, 512, 1))  # can never fit
    assert e.value.status == 7  # MC_ERR_BUDGET
    srv.close()
    mcpt.free_scene(s)


def test_guided_and_plain_requests_together(ctx):
    s, d = _scene(24, 4000)
    srv = mcpt.Server(ctx, samples_per_step=4)
    sid = srv.add_scene(d)
    g = srv.submit(sid, _params(s, 64, 8), guided=True)
    g2 = srv.submit(sid, _params(s, 48, 6), guided=True)  # shares the first one's waves and guide
    p = srv.submit(sid, _params(s, 64, 8))
    _drain(srv)
    for rid, W, spp in ((g, 64, 8), (g2, 48, 6), (p, 64, 8)):
        r = srv.result(rid)
        assert r.state == mcpt.REQ_DONE and r.spp_done == spp
        host = srv.read(rid, W, W)
        assert np.isfinite(host).all() and host.sum() > 0
    assert srv.stats().rays > 0
    srv.close()
    mcpt.free_scene(s)
