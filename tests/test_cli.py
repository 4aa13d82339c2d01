"""The `monocuda` command-line driver (reference flags over the C ABI)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import mcpt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "monocuda-pt_b200", "monocuda")


def _run(*args):
    return subprocess.run([CLI] + list(args), capture_output=True, text=True, timeout=300)


def _read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline().strip() == b"PF"
        w, h = map(int, f.readline().split())
        scale = float(f.readline())
        data = np.frombuffer(f.read(), dtype="<f4" if scale < 0 else ">f4")
    return data.reshape(h, w, 3)[::-1]  # PFM stores the bottom row first


@pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built")
def test_usage_errors_exit_2():
    r = _run("--bogus")
    assert r.returncode == 2 and "unknown argument" in r.stderr
    r = _run("--scene", "no_such_scene")
    assert r.returncode == 2 and "unknown scene" in r.stderr
    r = _run("--help")
    assert r.returncode == 0 and "--persistent" in r.stdout


@pytest.mark.gpu
def test_cli_render_equals_library_call(tmp_path):
    out = os.path.join(tmp_path, "c.pfm")
    r = _run("--wavefront", "--persistent", "--scene", "cornell_boxes", "--width", "64", "--spp", "2", "--stats",
             "--out", out)
    assert r.returncode == 0, r.stderr
    assert "Mrays/s" in r.stdout and "bounce 0" in r.stdout
    img = _read_pfm(out)
    assert img.shape == (64, 64, 3) and float(img.sum()) > 0

    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = 64
    cam.aspect_ratio = 1.0
    mcpt.camera_initialize(cam)
    p = mcpt.render_params(cam, 64, 64, 2, s.max_depth, persistent=True, rng=mcpt.RNG_PHILOX, seed=1234)
    ctx = mcpt.Context(0)
    tris = mcpt.host_triangles(s)
    acc = np.zeros(64 * 64 * 3, np.float32)
    env = mcpt.EnvMap()
    st = mcpt.RenderStats()
    mcpt.check(ctx.lib.mc_render_host(ctx.handle, C.addressof(tris), len(tris), None, 0, C.byref(env), C.byref(p),
                                      acc.ctypes.data, C.byref(st)))
    ctx.close()
    mcpt.free_scene(s)
    np.testing.assert_allclose(img.reshape(-1), acc / np.float32(2), rtol=4e-7, atol=0)


@pytest.mark.gpu
def test_cli_png_and_ppm_match_reference_resolve(tmp_path):
    """--tonemap aces --exposure 0.8: the PNG and PPM pixels equal the
    reference's resolve_kernel + 8-bit encoding of the same accumulation."""
    import mcref
    from test_cpu import _png_pixels
    outs = [os.path.join(tmp_path, "c.png"), os.path.join(tmp_path, "c.ppm")]
    for out in outs:
        r = _run("--wavefront", "--persistent", "--scene", "cornell_boxes", "--width", "48", "--spp", "3",
                 "--tonemap", "aces", "--exposure", "0.8", "--out", out)
        assert r.returncode == 0, r.stderr
    w, h, png = _png_pixels(open(outs[0], "rb").read())
    assert (w, h) == (48, 48)
    ppm = open(outs[1], "rb").read()
    assert ppm.startswith(b"P6\n48 48\n255\n")
    assert ppm[len(b"P6\n48 48\n255\n"):] == png.tobytes()

    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = 48
    cam.aspect_ratio = 1.0
    mcpt.camera_initialize(cam)
    p = mcpt.render_params(cam, 48, 48, 3, s.max_depth, persistent=True, rng=mcpt.RNG_PHILOX, seed=1234)
    ctx = mcpt.Context(0)
    tris = mcpt.host_triangles(s)
    acc = np.zeros(48 * 48 * 3, np.float32)
    env = mcpt.EnvMap()
    mcpt.check(ctx.lib.mc_render_host(ctx.handle, C.addressof(tris), len(tris), None, 0, C.byref(env), C.byref(p),
                                      acc.ctypes.data, None))
    ctx.close()
    mcpt.free_scene(s)
    rgb8 = np.zeros(48 * 48 * 3, np.uint8)
    assert mcref.load(False).mcref_resolve(acc.ctypes.data, 48, 48, 3, mcpt.TONEMAP_ACES, 0.8, 0, None,
                                           rgb8.ctypes.data, None) == 0
    assert np.array_equal(png.reshape(-1), rgb8)


def _sky(path, w=64, h=32):
    """A smooth sky as a PFM file (bottom row first); returns its RGBA, top row first."""
    y, x = np.meshgrid(np.linspace(0, 1, h), np.linspace(0, 1, w), indexing="ij")
    rgb = np.stack([0.3 + 2.0 * (1 - y) * (0.5 + 0.5 * np.sin(6 * x)), 0.4 + 1.5 * (1 - y), 0.9 + y * 0.2], -1)
    rgb = rgb.astype(np.float32)
    with open(path, "wb") as f:
        f.write(b"PF\n%d %d\n-1.0\n" % (w, h) + rgb[::-1].astype("<f4").tobytes())
    return np.concatenate([rgb, np.ones((h, w, 1), np.float32)], -1)


@pytest.mark.gpu
def test_cli_environment_map_matches_reference(tmp_path):
    """--env FILE.pfm --env-intensity 0.7 --env-rotation 30: the linear image
    equals the reference's render with the same map, intensity and rotation."""
    import mcref
    from test_gpu_parity import pixel_agreement
    sky = _sky(os.path.join(tmp_path, "sky.pfm"))
    out = os.path.join(tmp_path, "e.pfm")
    r = _run("--wavefront", "--persistent", "--scene", "displaced_icospheres", "--variant", "5", "--width", "160",
             "--spp", "2", "--env", os.path.join(tmp_path, "sky.pfm"), "--env-intensity", "0.7", "--env-rotation", "30",
             "--out", out)
    assert r.returncode == 0, r.stderr
    assert "Environment map" in r.stdout
    img = _read_pfm(out)
    s = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=5)
    H = s.height * 160 // s.width
    tris = mcpt.host_triangles(s)
    ref = mcref.load(True)
    assert ref.mcref_scene_upload(C.addressof(tris), len(tris), None, 0, sky.ctypes.data, 64, 32, 0.7, 30.0) == 0
    acc = np.zeros(160 * H * 3, np.float32)
    stats = np.zeros(3, np.float64)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    assert ref.mcref_render(C.addressof(cam), 160, H, 2, s.max_depth, 2, 1234, 0, 0, acc.ctypes.data,
                            stats.ctypes.data) == 0
    want = acc.reshape(H, 160, 3) / np.float32(2)
    frac = pixel_agreement(img, want)
    print("environment map: pixel agreement %.6f" % frac)
    assert frac >= 0.999
    mcpt.free_scene(s)


@pytest.mark.gpu
def test_cli_volume_and_phase_g_equal_library_render(tmp_path):
    """--volume FILE --phase-g 0.5 on the spheres scene: the grid fills its
    medium sphere and the image equals the library's render of the same."""
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_SPHERES)
    sp = mcpt.host_spheres(s)[1]
    c = np.array([sp.center.x, sp.center.y, sp.center.z], np.float32)
    d, org = mcpt.fog_sphere(sp.radius, sp.radius / 8.0)
    grid_path = os.path.join(tmp_path, "fog.mcvol")
    mcpt.volume_file_write(grid_path, d, tuple(np.asarray(org, np.float32) + c), sp.radius / 8.0)
    out = os.path.join(tmp_path, "v.pfm")
    r = _run("--wavefront", "--persistent", "--scene", "cornell_spheres", "--width", "64", "--spp", "2",
             "--volume", grid_path, "--phase-g", "0.5", "--out", out)
    assert r.returncode == 0, r.stderr
    assert "1 medium primitives" in r.stdout
    img = _read_pfm(out)

    ctx = mcpt.Context(0)
    dens, origin, voxel = mcpt.volume_file_read(grid_path)
    g, h = mcpt.volume_grid_create(ctx, dens, origin, voxel)
    sp.mat.density_grid = g
    sp.mat.grid_max_density = h.maximum_density
    sp.mat.phase_g = 0.5
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = 64
    cam.aspect_ratio = 1.0
    mcpt.camera_initialize(cam)
    p = mcpt.render_params(cam, 64, 64, 2, s.max_depth, persistent=True, rng=mcpt.RNG_PHILOX, seed=1234)
    tris = mcpt.host_triangles(s)
    sph = mcpt.host_spheres(s)
    acc = np.zeros(64 * 64 * 3, np.float32)
    env = mcpt.EnvMap()
    st = mcpt.RenderStats()
    mcpt.check(ctx.lib.mc_render_host(ctx.handle, C.addressof(tris), len(tris), C.addressof(sph), len(sph), C.byref(env),
                                      C.byref(p), acc.ctypes.data, C.byref(st)))
    mcpt.volume_grid_destroy(g)
    ctx.close()
    mcpt.free_scene(s)
    assert st.error_flags == 0
    np.testing.assert_allclose(img.reshape(-1), acc / np.float32(2), rtol=4e-7, atol=0)


@pytest.mark.gpu
def test_cli_cloud_scene(tmp_path):
    """--scene cloud --volume FILE: the reference's cloud set-up around the
    grid renders (deep paths, roulette cap 0.95)."""
    d, org = mcpt.fog_sphere(60.0, 4.0)
    path = os.path.join(tmp_path, "cloud.mcvol")
    mcpt.volume_file_write(path, d, tuple(np.asarray(org, np.float32) + np.float32([0, 100, -40])), 4.0)
    out = os.path.join(tmp_path, "cloud.pfm")
    r = _run("--wavefront", "--persistent", "--scene", "cloud", "--volume", path, "--width", "96", "--spp", "1",
             "--out", out)
    assert r.returncode == 0, r.stderr
    assert "1 medium primitives" in r.stdout and "depth 1000" in r.stdout
    img = _read_pfm(out)
    assert img.shape == (51, 96, 3) and np.isfinite(img).all() and float(img.mean()) > 0
