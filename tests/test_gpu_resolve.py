"""Resolve and output encoding (mc_image_encode, mc_server_encode) against the
reference's resolve_kernel and computeAutoExposure, run from oracle/_ref on
the same GPU, and main()'s 8-bit encoding (PT:3060-3132, 4363-4380).

Bars: with a given exposure the frame buffer floats and the 8-bit pixels are
bit-exact. With the automatic exposure the reference adds FP32 warp sums with
atomics in no fixed order and the library sums in FP64 in a fixed order: the
exposure agrees within 2e-5 relative, the floats within 1e-4 relative and
the bytes within 1 (at least 99 % identical).
"""
import ctypes as C

import numpy as np
import pytest

import mcpt
import mcref

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = mcpt.Context(0)
    yield c
    c.close()


def accum_image(w, h, samples, seed):
    """Sums over `samples` samples: log-normal radiance with a few negative,
    NaN and infinite pixels, as an accumulation buffer can hold."""
    rng = np.random.default_rng(seed)
    a = (rng.lognormal(-1.0, 1.5, (h, w, 3)) * samples).astype(np.float32)
    flat = a.reshape(-1)
    k = max(1, flat.size // 5000)
    idx = rng.choice(flat.size, 3 * k, replace=False)
    flat[idx[:k]] = -flat[idx[:k]]
    if w * h > 1:
        flat[idx[k:2 * k]] = np.nan
        flat[idx[2 * k:]] = np.inf
    return a.reshape(-1)


def reference(accum, w, h, samples, tonemap, exposure):
    frame = np.zeros(w * h * 3, np.float32)
    rgb8 = np.zeros(w * h * 3, np.uint8)
    chosen = C.c_float()
    auto = 1 if exposure <= 0 else 0
    assert mcref.load(False).mcref_resolve(accum.ctypes.data, w, h, samples, tonemap, exposure if not auto else 1.0,
                                           auto, frame.ctypes.data, rgb8.ctypes.data, C.byref(chosen)) == 0
    return frame, rgb8, chosen.value


SIZES = [(1, 1), (17, 13), (640, 480), (1920, 1080)]


@pytest.mark.parametrize("w,h", SIZES)
@pytest.mark.parametrize("tonemap", [mcpt.TONEMAP_NONE, mcpt.TONEMAP_REINHARD, mcpt.TONEMAP_ACES])
@pytest.mark.parametrize("exposure", [1.0, 0.37, 0.0])
def test_resolve_matches_reference(ctx, w, h, tonemap, exposure):
    samples = 16
    accum = accum_image(w, h, samples, seed=w + 7 * h + tonemap)
    if exposure <= 0:
        accum = np.nan_to_num(accum, nan=1.0, posinf=2.0)  # the auto exposure of a NaN pixel is tested below
    d = torch.from_numpy(accum).cuda()
    f32, e_f = mcpt.image_encode(ctx, d.data_ptr(), w, h, samples, mcpt.IMAGE_RGB_F32, tonemap, exposure)
    b8, e_b = mcpt.image_encode(ctx, d.data_ptr(), w, h, samples, mcpt.IMAGE_RGB8, tonemap, exposure)
    frame = np.frombuffer(f32, np.float32)
    rgb8 = np.frombuffer(b8, np.uint8)
    rf, r8, re = reference(accum, w, h, samples, tonemap, exposure)
    assert e_f == e_b
    if exposure > 0:
        assert e_f == np.float32(exposure)
        assert np.array_equal(frame.view(np.uint32), rf.view(np.uint32)), "frame buffer differs from resolve_kernel"
        assert np.array_equal(rgb8, r8), "8-bit pixels differ from main()'s encoding"
    else:
        assert abs(e_f - re) <= 2e-5 * abs(re), (e_f, re)
        fin = np.isfinite(rf)
        assert np.array_equal(fin, np.isfinite(frame))
        assert np.allclose(frame[fin], rf[fin], rtol=1e-4, atol=1e-6)
        diff = np.abs(rgb8.astype(np.int32) - r8.astype(np.int32))
        assert diff.max() <= 1 and (diff == 0).mean() >= 0.99


def test_auto_exposure_ignores_nan_and_inf_luminance(ctx):
    w, h, samples = 257, 129, 4
    accum = accum_image(w, h, samples, seed=5)
    d = torch.from_numpy(accum).cuda()
    _, e = mcpt.image_encode(ctx, d.data_ptr(), w, h, samples, mcpt.IMAGE_RGB8, mcpt.TONEMAP_ACES, 0.0)
    _, _, re = reference(accum, w, h, samples, mcpt.TONEMAP_ACES, 0.0)
    assert np.isfinite(e) and abs(e - re) <= 2e-5 * abs(re)


def test_auto_exposure_is_deterministic(ctx):
    w, h, samples = 1920, 1080, 64
    accum = np.nan_to_num(accum_image(w, h, samples, seed=3), nan=0.0, posinf=0.0)
    d = torch.from_numpy(accum).cuda()
    outs = [mcpt.image_encode(ctx, d.data_ptr(), w, h, samples, mcpt.IMAGE_RGB8, mcpt.TONEMAP_REINHARD, 0.0)
            for _ in range(3)]
    assert all(o == outs[0] for o in outs)


def test_pfm_and_png_outputs(ctx):
    w, h, samples, exposure = 33, 21, 8, 0.5
    accum = accum_image(w, h, samples, seed=9)
    d = torch.from_numpy(accum).cuda()
    pfm, _ = mcpt.image_encode(ctx, d.data_ptr(), w, h, samples, mcpt.IMAGE_PFM, mcpt.TONEMAP_ACES, exposure)
    header = b"PF\n%d %d\n-1.0\n" % (w, h)
    assert pfm.startswith(header) and len(pfm) == len(header) + w * h * 12
    rows = np.frombuffer(pfm[len(header):], np.float32).reshape(h, w, 3)[::-1]  # PFM: bottom row first
    want = (accum.reshape(h, w, 3) / np.float32(samples)) * np.float32(exposure)
    fin = np.isfinite(want)
    assert np.array_equal(fin, np.isfinite(rows))
    assert np.allclose(rows[fin], want[fin], rtol=4e-7, atol=0)  # linear radiance, no tone map (fast-math division)
    png, _ = mcpt.image_encode(ctx, d.data_ptr(), w, h, samples, mcpt.IMAGE_PNG, mcpt.TONEMAP_ACES, exposure)
    from test_cpu import _png_pixels
    gw, gh, px = _png_pixels(png)
    _, r8, _ = reference(accum, w, h, samples, mcpt.TONEMAP_ACES, exposure)
    assert (gw, gh) == (w, h) and np.array_equal(px.reshape(-1), r8)


def test_device_output_equals_host_output(ctx):
    w, h, samples = 640, 360, 4
    accum = accum_image(w, h, samples, seed=13)
    d = torch.from_numpy(accum).cuda()
    host8, _ = mcpt.image_encode(ctx, d.data_ptr(), w, h, samples, mcpt.IMAGE_RGB8, mcpt.TONEMAP_ACES, 1.5)
    dev8 = torch.zeros(w * h * 3, dtype=torch.uint8, device="cuda")
    mcpt.image_encode(ctx, d.data_ptr(), w, h, samples, mcpt.IMAGE_RGB8, mcpt.TONEMAP_ACES, 1.5,
                      device_out=dev8.data_ptr())
    assert dev8.cpu().numpy().tobytes() == host8


def test_encode_rejects_bad_options(ctx):
    d = torch.zeros(12, dtype=torch.float32, device="cuda")
    lib = mcpt.load()
    n = C.c_int64(1 << 20)
    out = (C.c_uint8 * (1 << 20))()
    for fmt, tm, dev in [(7, 0, 0), (0, 9, 0), (mcpt.IMAGE_PNG, 0, 1), (mcpt.IMAGE_PFM, 0, 1)]:
        o = mcpt.ImageOptions(fmt, tm, 1.0, dev)
        assert lib.mc_image_encode(ctx.handle, d.data_ptr(), 2, 2, 1, C.byref(o), out, C.byref(n), None) == 1
    o = mcpt.ImageOptions(mcpt.IMAGE_RGB8, 0, 1.0, 0)
    small = C.c_int64(5)
    assert lib.mc_image_encode(ctx.handle, d.data_ptr(), 2, 2, 1, C.byref(o), out, C.byref(small), None) == 1
    assert lib.mc_image_encode(ctx.handle, d.data_ptr(), 2, 2, 0, C.byref(o), out, C.byref(n), None) == 1


def test_server_encodes_finished_request(ctx):
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES, seed=2)
    ds = mcpt.DeviceScene(mcpt.host_triangles(s))
    srv = mcpt.Server(ctx, samples_per_step=4)
    sid = srv.add_scene(ds)
    w, h, spp = 96, 64, 8
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = w
    cam.aspect_ratio = w / h
    mcpt.camera_initialize(cam)
    p = mcpt.render_params(cam, w, h, spp, 8)
    rid = srv.submit(sid, p)
    for _ in range(100):
        srv.step()
        if srv.result(rid).state == mcpt.REQ_DONE:
            break
    assert srv.result(rid).state == mcpt.REQ_DONE
    acc = srv.read(rid, w, h)
    for tm, ex in [(mcpt.TONEMAP_ACES, 1.0), (mcpt.TONEMAP_NONE, 0.0)]:
        got, chosen = srv.encode(rid, mcpt.IMAGE_RGB8, tm, ex)
        _, r8, re = reference(acc, w, h, spp, tm, ex)
        g = np.frombuffer(got, np.uint8)
        if ex > 0:
            assert np.array_equal(g, r8)
        else:
            assert abs(chosen - re) <= 2e-5 * abs(re)
            assert np.abs(g.astype(int) - r8.astype(int)).max() <= 1
    pfm, _ = srv.encode(rid, mcpt.IMAGE_PFM, mcpt.TONEMAP_NONE, 1.0)
    assert pfm.startswith(b"PF\n96 64\n-1.0\n")
    srv.release(rid)
    srv.close()
    mcpt.free_scene(s)
