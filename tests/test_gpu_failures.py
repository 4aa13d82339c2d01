"""Failure paths of the device error word, made without faulting the GPU.

The reference stops the process on any CUDA error (PT:55-63) and has no
bounded waits, stack or queue checks that report back. Here every one of
these becomes an mc_status and the context stays usable:
  * a bounded wait on a flag that nothing sets runs out -> MC_ERR_TIMEOUT;
  * a queue capacity too small for the wave -> MC_ERR_QUEUE_OVERFLOW (the
    excess entries are dropped, nothing is written past the capacity);
  * a traversal stack limit below what the tree needs -> MC_ERR_STACK_OVERFLOW
    (the ray is abandoned, nothing is written past the limit);
  * a server request cancelled between steps -> MC_ERR_CANCELLED on reads,
    its memory back in the budget, the other requests unaffected.
After each failure an ordinary render on the same context gives the image a
fresh context gives.
"""
import ctypes as C

import numpy as np
import pytest

import mcpt

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

OK, STACK, QUEUE, TIMEOUT, CANCELLED, INVALID = 0, 4, 5, 6, 8, 1


@pytest.fixture(scope="module")
def ctx():
    c = mcpt.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def cornell():
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
    return s, mcpt.DeviceScene(mcpt.host_triangles(s))


def _params(s, W, spp, **kw):
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = 1.0
    mcpt.camera_initialize(cam)
    return mcpt.render_params(cam, W, W, spp, 8, persistent=True, rng=mcpt.RNG_PHILOX, seed=3, **kw)


def _render(ctx, bvh, d, p):
    acc = torch.zeros(p.width * p.height * 3, dtype=torch.float32, device="cuda")
    st = mcpt.RenderStats()
    status = ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(d.view), C.byref(p), acc.data_ptr(),
                                         C.byref(st))
    return status, acc.cpu().numpy(), st


def _fresh_reference(s, d, W, spp, layout=mcpt.LAYOUT_WIDE4):
    c2 = mcpt.Context(0)
    b2 = mcpt.Bvh(c2, d.view, layout=layout)
    status, img, _ = _render(c2, b2, d, _params(s, W, spp))
    assert status == OK
    b2.close()
    c2.close()
    return img


def test_wait_on_a_flag_nothing_sets_times_out(ctx, cornell):
    s, d = cornell
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    mcpt.check(ctx.lib.mc_context_set_wait_timeout(ctx.handle, 2000))  # 2 ms
    mcpt.check(ctx.lib.mc_stream_wait_value(ctx.handle, flag.data_ptr(), 1))
    assert ctx.lib.mc_context_synchronize(ctx.handle) == TIMEOUT
    assert b"wait timeout" in ctx.lib.mc_last_error()
    # reported once, then cleared
    assert ctx.lib.mc_context_synchronize(ctx.handle) == OK
    # the flag is set: the wait passes
    flag.fill_(1)
    torch.cuda.synchronize()
    mcpt.check(ctx.lib.mc_stream_wait_value(ctx.handle, flag.data_ptr(), 1))
    assert ctx.lib.mc_context_synchronize(ctx.handle) == OK
    mcpt.check(ctx.lib.mc_context_set_wait_timeout(ctx.handle, 0))
    # the context renders as a fresh one does
    bvh = mcpt.Bvh(ctx, d.view, layout=mcpt.LAYOUT_WIDE4)
    status, img, _ = _render(ctx, bvh, d, _params(s, 64, 2))
    assert status == OK
    assert np.array_equal(img, _fresh_reference(s, d, 64, 2))
    assert ctx.lib.mc_context_set_wait_timeout(ctx.handle, -1) == INVALID


def test_tiny_queue_capacity_reports_overflow(ctx, cornell):
    s, d = cornell
    bvh = mcpt.Bvh(ctx, d.view, layout=mcpt.LAYOUT_WIDE4)
    for cap in (100, 4095):
        status, img, st = _render(ctx, bvh, d, _params(s, 64, 1, queue_capacity=cap))
        assert status == QUEUE, cap
        assert b"capacity" in ctx.lib.mc_last_error()
        assert st.error_flags & 2
        assert np.isfinite(img).all()
    # a capacity that holds every path is no overflow, and the images agree
    status, img, _ = _render(ctx, bvh, d, _params(s, 64, 2, queue_capacity=64 * 64))
    assert status == OK
    status, img2, _ = _render(ctx, bvh, d, _params(s, 64, 2))
    assert status == OK and np.array_equal(img, img2)
    assert np.array_equal(img2, _fresh_reference(s, d, 64, 2))


@pytest.mark.parametrize("layout", [mcpt.LAYOUT_BINARY, mcpt.LAYOUT_WIDE4])
def test_stack_limit_below_the_tree_reports_overflow(ctx, layout):
    s = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=5, seed=2)
    d = mcpt.DeviceScene(mcpt.host_triangles(s))
    bvh = mcpt.Bvh(ctx, d.view, layout=layout)
    status, img, st = _render(ctx, bvh, d, _params(s, 48, 1, stack_entries=2))
    assert status == STACK
    assert st.error_flags & 1
    assert np.isfinite(img).all()
    # a limit the tree fits in (the full 64, and 48 for the 4-wide tree) renders the default image
    ref = _fresh_reference(s, d, 48, 2, layout=layout)
    for entries in (0, 64) + ((48,) if layout == mcpt.LAYOUT_WIDE4 else ()):
        status, img, _ = _render(ctx, bvh, d, _params(s, 48, 2, stack_entries=entries))
        assert status == OK, entries
        assert np.array_equal(img, ref), entries
    assert _render(ctx, bvh, d, _params(s, 48, 1, stack_entries=65))[0] == INVALID
    mcpt.free_scene(s)


def test_server_request_cancelled_mid_render(ctx, cornell):
    s, d = cornell
    srv = mcpt.Server(ctx, samples_per_step=2, max_active=2)
    sid = srv.add_scene(d)
    a = srv.submit(sid, _params(s, 64, 8))
    b = srv.submit(sid, _params(s, 48, 6))
    c = srv.submit(sid, _params(s, 32, 4))  # waits: two requests at a time
    srv.step()
    ra = srv.result(a)
    assert ra.state == mcpt.REQ_ACTIVE and ra.spp_done == 2
    used = srv.stats().used_bytes
    srv.cancel(a)
    ra = srv.result(a)
    assert ra.state == mcpt.REQ_CANCELLED and ra.spp_done == 2 and not ra.d_accum
    assert srv.stats().used_bytes == used - ra.bytes
    host = np.zeros(64 * 64 * 3, np.float32)
    assert ctx.lib.mc_server_read(srv.handle, a, host.ctypes.data) == CANCELLED
    assert ctx.lib.mc_server_cancel(srv.handle, a) == CANCELLED
    # a pending request is cancelled before it is ever admitted
    assert srv.result(c).state == mcpt.REQ_PENDING
    srv.cancel(c)
    assert srv.result(c).state == mcpt.REQ_CANCELLED and srv.result(c).spp_done == 0
    for _ in range(100):
        if srv.step() == 0 and srv.stats().pending == 0:
            break
    rb = srv.result(b)
    assert rb.state == mcpt.REQ_DONE and rb.spp_done == 6
    assert ctx.lib.mc_server_cancel(srv.handle, b) == INVALID
    # the request that stayed renders the image a standalone render gives
    assert np.array_equal(srv.read(b, 48, 48), _fresh_reference(s, d, 48, 6))
    srv.release(b)
    srv.release(a)  # a cancelled request holds nothing: releasing it is a no-op
    assert srv.stats().used_bytes == srv.stats().scene_bytes
