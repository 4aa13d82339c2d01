"""Heterogeneous media (mc_volume_grid on an isotropic material): delta
tracking in shade and ratio tracking of shadow rays, against the reference's
own heterogeneousFreeFlightDistance / heterogeneousTransmittance
(PT:796-838), run from oracle/_ref on the same grids (its nanovdb stand-in
reads the same dense layout). Bars as the other image-parity tests: per
pixel within 1e-4 relative for at least 99.9 % of the pixels, under the
counter-based Philox draws and under the reference's curand XORWOW.

A grid of constant value c with extinction scale s is a homogeneous medium
of density s*c: the images agree in expectation (within 4 standard errors).
"""
import ctypes as C

import numpy as np
import pytest

import mcpt
from test_gpu_parity import pixel_agreement, render_mine, render_ref

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = mcpt.Context(0)
    yield c
    c.close()


def trilinear(density, origin, voxel, pts):
    """The sampler's reading: index point (p - origin) * (1 / voxel) in
    float32 as the grid forms it, then the 8 voxels around its floor (0
    outside) interpolated in float64 along z, then y, then x."""
    nz, ny, nx = density.shape
    inv = np.float32(1.0) / np.float32(voxel)
    x = ((pts.astype(np.float32) - np.asarray(origin, np.float32)) * inv).astype(np.float64)
    f = np.floor(x)
    i = f.astype(np.int64)
    u = x - f

    def at(a, b, c):
        ok = (a >= 0) & (b >= 0) & (c >= 0) & (a < nx) & (b < ny) & (c < nz)
        v = np.zeros(len(a))
        v[ok] = density[c[ok], b[ok], a[ok]]
        return v

    def lerp(a, b, w):
        return a + w * (b - a)
    ix, iy, iz = i[:, 0], i[:, 1], i[:, 2]
    c00 = lerp(at(ix, iy, iz), at(ix, iy, iz + 1), u[:, 2])
    c01 = lerp(at(ix, iy + 1, iz), at(ix, iy + 1, iz + 1), u[:, 2])
    c10 = lerp(at(ix + 1, iy, iz), at(ix + 1, iy, iz + 1), u[:, 2])
    c11 = lerp(at(ix + 1, iy + 1, iz), at(ix + 1, iy + 1, iz + 1), u[:, 2])
    return lerp(lerp(c00, c01, u[:, 1]), lerp(c10, c11, u[:, 1]), u[:, 0])


def noise_grid(lo, hi, voxel, seed):
    """Smooth non-negative density over the box [lo, hi] (2 voxels of margin)."""
    rng = np.random.default_rng(seed)
    origin = np.asarray(lo, np.float64) - 2 * voxel
    n = np.ceil((np.asarray(hi) - origin) / voxel).astype(int) + 3
    z, y, x = np.meshgrid(*[origin[a] + voxel * np.arange(n[a]) for a in (2, 1, 0)], indexing="ij")
    d = np.zeros(x.shape)
    for _ in range(6):
        k = rng.normal(0, 3.0, 3)
        d += np.sin(k[0] * x + k[1] * y + k[2] * z + rng.uniform(0, 6.3)) * rng.uniform(0.2, 1.0)
    d = np.maximum(d, 0.0) + 0.05 * rng.random(d.shape)
    return d.astype(np.float32), tuple(origin.astype(np.float32))


def test_density_matches_trilinear_reading(ctx):
    d, org = noise_grid((-1, -0.5, 0.2), (0.8, 0.9, 1.5), 0.07, seed=3)
    g, h = mcpt.volume_grid_create(ctx, d, org, 0.07)
    assert h.maximum_density == d.max() and tuple(h.dims) == (d.shape[2], d.shape[1], d.shape[0])
    rng = np.random.default_rng(1)
    pts = rng.uniform((-1.3, -0.8, -0.1), (1.1, 1.2, 1.8), (200000, 3)).astype(np.float32)
    pts[:1000] = np.asarray(org, np.float32) + 0.07 * rng.integers(-2, 30, (1000, 3))  # voxel centres
    pts[1000:1010] = np.nan
    dp = torch.from_numpy(pts).cuda()
    out = torch.zeros(len(pts), dtype=torch.float32, device="cuda")
    mcpt.volume_density(ctx, g, dp, len(pts), out)
    got = out.cpu().numpy()
    fin = np.isfinite(pts).all(1)
    want = trilinear(d.astype(np.float64), org, 0.07, pts[fin])
    assert np.all(got[~fin] == 0)
    assert np.abs(got[fin] - want).max() <= 1e-6 * max(1.0, d.max())
    mcpt.volume_grid_destroy(g)


def test_create_rejects_bad_grids(ctx):
    lib = mcpt.load()
    o = (C.c_float * 3)(0, 0, 0)
    g = C.c_void_p()
    for bad in (np.full((2, 2, 2), -1, np.float32), np.full((2, 2, 2), np.nan, np.float32), np.zeros((2, 2, 2), np.float32)):
        assert lib.mc_volume_grid_create(ctx.handle, bad.ctypes.data, 2, 2, 2, o, 0.1, C.byref(g), None) == 1
    ok = np.ones((2, 2, 2), np.float32)
    assert lib.mc_volume_grid_create(ctx.handle, ok.ctypes.data, 2, 2, 2, o, 0.0, C.byref(g), None) == 1


_grids = []


def gridded_spheres(ctx, scale=3.0, constant=None):
    """The spheres scene with its medium sphere (sphere 1) filled by a fog
    sphere grid (or a constant grid covering it)."""
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_SPHERES, seed=2)
    sp = mcpt.host_spheres(s)[1]
    assert sp.mat.type == mcpt.MAT_ISOTROPIC
    c = np.array([sp.center.x, sp.center.y, sp.center.z], np.float32)
    voxel = sp.radius / 10.0
    if constant is None:
        d, org = mcpt.fog_sphere(sp.radius, voxel)
    else:
        n = 25
        d = np.full((n, n, n), constant, np.float32)
        org = tuple(-voxel * 12 for _ in range(3))
    g, h = mcpt.volume_grid_create(ctx, d, tuple(np.asarray(org, np.float32) + c), voxel)
    _grids.append(g)
    sp.mat.density = scale
    sp.mat.phase_g = 0.3
    sp.mat.density_grid = g
    sp.mat.grid_max_density = h.maximum_density
    return s


def gridded_box(ctx):
    """Displaced icospheres variant 5 with its medium box (12 isotropic
    triangles) filled by a smooth noise grid."""
    s = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=5, seed=2)
    tris = mcpt.host_triangles(s)
    raw = np.frombuffer(tris, np.uint8).reshape(len(tris), 224)
    iso = np.where(raw[:, 96:100].copy().view(np.int32).ravel() == mcpt.MAT_ISOTROPIC)[0]
    v = raw[iso, :36].copy().view(np.float32).reshape(-1, 3)
    d, org = noise_grid(v.min(0), v.max(0), 0.05, seed=11)
    g, h = mcpt.volume_grid_create(ctx, d, org, 0.05)
    _grids.append(g)
    for i in iso:
        tris[i].mat.density_grid = g
        tris[i].mat.grid_max_density = h.maximum_density
    return s


@pytest.mark.parametrize("layout", [mcpt.LAYOUT_BINARY, mcpt.LAYOUT_WIDE4])
@pytest.mark.parametrize("which", ["sphere", "box"])
def test_grid_medium_image_parity_philox(ctx, which, layout):
    s = gridded_spheres(ctx) if which == "sphere" else gridded_box(ctx)
    W, H, spp = (256, 256, 4) if which == "sphere" else (320, 180, 2)
    mine, st = render_mine(ctx, s, W, H, spp, 8, mcpt.RNG_PHILOX, env=which == "box", layout=layout)
    ref, rs = render_ref(s, W, H, spp, 8, 2, philox=True, env=which == "box")
    frac = pixel_agreement(mine, ref)
    print("%s layout %d: pixel agreement %.6f, identical %.6f" % (which, layout, frac,
                                                                 np.mean(np.all(mine == ref, axis=2))))
    assert st.error_flags == 0
    assert frac >= 0.999
    assert abs(st.extend_rays - rs[0]) <= 0.001 * rs[0]
    mcpt.free_scene(s)


def test_grid_medium_image_parity_xorwow_unmodified(ctx):
    """Against renderWithWavefront itself with curand XORWOW: the shadow
    kernel's ratio tracking draws from, and stores back, the pixel's state."""
    s = gridded_spheres(ctx)
    mine, _ = render_mine(ctx, s, 256, 256, 2, 8, mcpt.RNG_XORWOW)
    ref, _ = render_ref(s, 256, 256, 2, 8, 2, philox=False, unmodified=1)
    frac = pixel_agreement(mine, ref)
    print("xorwow pixel agreement %.6f" % frac)
    assert frac >= 0.999
    mcpt.free_scene(s)


def _render(ctx, s, W, H, spp, first, graph=False, flags=None):
    ds = mcpt.DeviceScene(mcpt.host_triangles(s), spheres=mcpt.host_spheres(s))
    if flags is not None:
        ds.view.has_medium = flags
    bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = W / float(H)
    mcpt.camera_initialize(cam)
    p = mcpt.render_params(cam, W, H, spp, 8, rng=mcpt.RNG_PHILOX, seed=5, first_sample=first, use_graph=graph)
    acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    st = mcpt.RenderStats()
    try:
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               C.byref(st)))
    finally:
        bvh.close()
    return acc.cpu().numpy(), ds.view.has_medium


def test_scene_flags_and_graph_replay(ctx):
    s = gridded_spheres(ctx)
    a, flags = _render(ctx, s, 96, 96, 4, 0)
    assert flags == mcpt.MEDIUM_ANY | mcpt.MEDIUM_GRID
    ds = mcpt.DeviceScene(mcpt.host_triangles(s), spheres=mcpt.host_spheres(s), ctx=ctx)
    assert ds.view.has_medium == mcpt.MEDIUM_ANY | mcpt.MEDIUM_GRID  # device ingestion reports it too
    b, _ = _render(ctx, s, 96, 96, 4, 0, graph=True)
    assert a.tobytes() == b.tobytes()
    # a grid in a scene view whose flags do not say so is an error, not a silent transparent medium
    with pytest.raises(mcpt.McError) as e:
        _render(ctx, s, 96, 96, 1, 0, flags=mcpt.MEDIUM_ANY)
    assert e.value.status == 1
    mcpt.free_scene(s)


def test_constant_grid_equals_homogeneous_medium_in_expectation(ctx):
    """Delta tracking through a constant grid accepts every tentative
    collision and ratio tracking returns 0 or 1: the same expectation as the
    homogeneous medium of density scale * c."""
    W = 64
    homog = mcpt.generate_scene(mcpt.SCENE_CORNELL_SPHERES, seed=2)
    mcpt.host_spheres(homog)[1].mat.density = 2.0
    mcpt.host_spheres(homog)[1].mat.phase_g = 0.3  # as gridded_spheres sets it
    grid = gridded_spheres(ctx, scale=4.0, constant=0.5)
    means = {}
    for name, s in (("homogeneous", homog), ("grid", grid)):
        means[name] = np.array([_render(ctx, s, W, W, 64, 1000 + 64 * b)[0].reshape(-1, 3).mean(0) for b in range(8)])
    h, g = means["homogeneous"], means["grid"]
    se = np.sqrt(h.var(0, ddof=1) / len(h) + g.var(0, ddof=1) / len(g))
    diff = np.abs(h.mean(0) - g.mean(0))
    print("means", h.mean(0), g.mean(0), "se", se)
    assert np.all(diff < 4 * se + 1e-6)
    mcpt.free_scene(homog)
    mcpt.free_scene(grid)


@pytest.mark.parametrize("grid", [True, False])
def test_paths_deeper_than_the_counter_block(ctx, grid):
    """Renders deeper than the 64 per-bounce counter slots (the cloud scene's
    max_depth is 1000, PT:4166): a dense medium with roulette capped at 0.95
    and max_depth 300 gives the reference's image and ray counts, and the
    deepest statistics bucket (depth 63 and deeper) is reached."""
    if grid:
        s = gridded_spheres(ctx, scale=60.0)
    else:
        s = mcpt.generate_scene(mcpt.SCENE_CORNELL_SPHERES, seed=2)
        mcpt.host_spheres(s)[1].mat.density = 40.0
    sp = mcpt.host_spheres(s)[1]
    sp.mat.albedo.color_a = mcpt.Vec3(1.0, 1.0, 1.0)
    s.camera.rr_cap = 0.95
    mine, st = render_mine(ctx, s, 128, 128, 2, 300, mcpt.RNG_PHILOX, layout=mcpt.LAYOUT_WIDE4)
    ref, rs = render_ref(s, 128, 128, 2, 300, 2, philox=True)
    frac = pixel_agreement(mine, ref)
    print("deep (grid %s): pixel agreement %.6f, rays %d+%d (reference %d+%d), depth 63+ extend %d"
          % (grid, frac, st.extend_rays, st.shadow_rays, rs[0], rs[1], st.extend_per_depth[63]))
    assert st.error_flags == 0
    assert frac >= 0.999
    assert abs(st.extend_rays - rs[0]) <= 0.001 * rs[0]
    assert st.extend_per_depth[63] > 0
    assert st.extend_rays == sum(st.extend_per_depth[i] for i in range(64))
    mcpt.free_scene(s)



def _fog_cloud(ctx, radius=60.0, voxel=4.0, centre=(0.0, 100.0, -40.0)):
    d, org = mcpt.fog_sphere(radius, voxel)
    g, h = mcpt.volume_grid_create(ctx, d, tuple(np.asarray(org, np.float32) + np.asarray(centre, np.float32)), voxel)
    _grids.append(g)
    return g, h


def test_cloud_scene_image_parity(ctx):
    """The reference's cloud scene (mc_scene_cloud: enclosing medium sphere,
    ground, sun quad, the Mitsuba camera, max depth 1000, roulette cap 0.95)
    around a fog-sphere grid: image and ray counts equal the reference's
    render of the same primitives and grid."""
    g, h = _fog_cloud(ctx)
    s = mcpt.SceneHost()
    mcpt.check(ctx.lib.mc_scene_cloud(g, C.byref(h), 1, C.byref(s)))
    assert s.max_depth == 1000 and s.camera.rr_cap == np.float32(0.95)
    W = 96
    H = 180 * W // 333
    mine, st = render_mine(ctx, s, W, H, 2, s.max_depth, mcpt.RNG_PHILOX, layout=mcpt.LAYOUT_WIDE4)
    ref, rs = render_ref(s, W, H, 2, s.max_depth, 2, philox=True)
    frac = pixel_agreement(mine, ref)
    print("cloud: pixel agreement %.6f, rays %d+%d (reference %d+%d), depth 63+ extend %d, mean %.4f"
          % (frac, st.extend_rays, st.shadow_rays, rs[0], rs[1], st.extend_per_depth[63], float(mine.mean())))
    assert st.error_flags == 0 and float(mine.mean()) > 0
    assert frac >= 0.999
    assert abs(st.extend_rays - rs[0]) <= 0.001 * rs[0]
    mcpt.free_scene(s)



def test_grid_scene_in_a_batch_equals_its_single_render(ctx):
    """A gridded scene batched with a plain one (shared waves, per-path scene
    ids, ratio tracking on each path's own scene): both images equal their
    single-scene renders."""
    scenes = [gridded_spheres(ctx), mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)]
    devs = [mcpt.DeviceScene(mcpt.host_triangles(s), spheres=mcpt.host_spheres(s)) for s in scenes]
    assert devs[0].view.has_medium & mcpt.MEDIUM_GRID and not devs[1].view.has_medium
    batch = mcpt.BatchBvh(ctx, [d.view for d in devs], layout=mcpt.LAYOUT_WIDE4)

    def params(s, W, spp):
        cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
        cam.image_width = W
        cam.aspect_ratio = 1.0
        mcpt.camera_initialize(cam)
        return mcpt.render_params(cam, W, W, spp, 8, rng=mcpt.RNG_PHILOX, seed=99)
    sizes = [(96, 3), (64, 2)]
    accs = [torch.zeros(W * W * 3, dtype=torch.float32, device="cuda") for W, _ in sizes]
    items = [mcpt.BatchItem(d.view, params(s, W, spp), a.data_ptr()) for d, s, a, (W, spp) in zip(devs, scenes, accs, sizes)]
    st = batch.render(items)
    assert st.error_flags == 0
    batch.close()
    for d, s, a, (W, spp) in zip(devs, scenes, accs, sizes):
        single = mcpt.Bvh(ctx, d.view, layout=mcpt.LAYOUT_WIDE4)
        ref = torch.zeros_like(a)
        rs = mcpt.RenderStats()
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, single.handle, C.byref(d.view), C.byref(params(s, W, spp)),
                                               ref.data_ptr(), C.byref(rs)))
        single.close()
        assert torch.equal(a, ref)
        assert float(a.sum()) > 0
    for s in scenes:
        mcpt.free_scene(s)



def test_release_grids(ctx):
    while _grids:
        mcpt.volume_grid_destroy(_grids.pop())
