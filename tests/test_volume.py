"""Density grids on the host (no GPU): the fog sphere of
createFogSphereGrid (src/volume_io.cpp:53-64) as mc_volume_fog_sphere builds
it, the grid header's layout, and argument checks."""
import ctypes as C

import numpy as np
import pytest

import mcpt


def test_header_layout():
    assert C.sizeof(mcpt.VolumeGrid) == 64
    assert mcpt.VolumeGrid.maximum_density.offset == 32 and mcpt.VolumeGrid.world_max.offset == 48
    # the material's grid fields sit where the reference's densityGrid / gridMaximumDensity do (PT:484-496)
    assert mcpt.Material.density_grid.offset == 80 and mcpt.Material.grid_max_density.offset == 88


def test_fog_sphere_values():
    r, h, band = 1.3, 0.1, 3.0
    d, org = mcpt.fog_sphere(r, h, band)
    r, h = float(np.float32(r)), float(np.float32(h))  # the library widens its float arguments
    n = d.shape[0]
    half = int(np.ceil(r / h)) + 1
    assert d.shape == (n, n, n) and n == 2 * half + 1
    assert np.allclose(org, -half * h)
    c = (np.arange(n) - half) * h
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    want = np.clip((r - np.sqrt(x * x + y * y + z * z)) / (band * h), 0.0, 1.0).astype(np.float32)
    assert np.array_equal(d, want)
    assert d[half, half, half] == 1.0 and d[0, 0, 0] == 0.0 and d.max() == 1.0
    # symmetric under every axis flip and axis swap
    assert np.array_equal(d, d[::-1]) and np.array_equal(d, d[:, ::-1]) and np.array_equal(d, d.transpose(2, 1, 0))
    # the ramp: strictly between 0 and 1 only within band * voxel inside the surface
    dist = np.sqrt(x * x + y * y + z * z)
    ramp = (d > 0) & (d < 1)
    assert np.all(dist[ramp] > r - band * h - 1e-9) and np.all(dist[ramp] < r + 1e-9)


def test_fog_sphere_rejects_bad_arguments():
    lib = mcpt.load()
    dims = (C.c_int32 * 3)()
    org = (C.c_float * 3)()
    for r, h, b in ((0.0, 0.1, 3.0), (1.0, 0.0, 3.0), (1.0, 0.1, 0.0), (float("nan"), 0.1, 3.0), (1.0, 1e-5, 3.0)):
        assert lib.mc_volume_fog_sphere(r, h, b, None, dims, org) == 1


def test_medium_flags_of_host_scenes():
    """The flags DeviceScene derives on the host path, as ingestion reports
    them: none, an isotropic medium, and one that carries a grid."""
    boxes = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
    spheres = mcpt.generate_scene(mcpt.SCENE_CORNELL_SPHERES)
    ico = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=5)
    f = mcpt._medium_flags
    assert f(mcpt.host_triangles(boxes), boxes.triangle_count, mcpt.Triangle) == 0
    sph = mcpt.host_spheres(spheres)
    assert f(sph, spheres.sphere_count, mcpt.Sphere) == mcpt.MEDIUM_ANY
    tris = mcpt.host_triangles(ico)
    assert f(tris, ico.triangle_count, mcpt.Triangle) == mcpt.MEDIUM_ANY
    sph[1].mat.density_grid = 0x1000  # any non-null pointer marks a grid; nothing is read through it here
    assert f(sph, spheres.sphere_count, mcpt.Sphere) == mcpt.MEDIUM_ANY | mcpt.MEDIUM_GRID
    sph[1].mat.density_grid = None
    sph[0].mat.density_grid = 0x1000  # a grid on a non-medium material is ignored, as ingestion ignores it
    assert f(sph, spheres.sphere_count, mcpt.Sphere) == mcpt.MEDIUM_ANY
    for s in (boxes, spheres, ico):
        mcpt.free_scene(s)


def _mat(m):
    return (bytes(C.c_int32(m.type)) + bytes(C.c_int32(m.albedo.type)) + bytes(m.albedo.color_a) + bytes(m.albedo.color_b)
            + bytes(C.c_float(m.albedo.scale)) + bytes(C.c_uint64(m.albedo.image)) + bytes(m.emitted)
            + bytes(C.c_float(m.fuzz)) + bytes(C.c_float(m.refraction_index)) + bytes(C.c_float(m.density))
            + bytes(C.c_float(m.phase_g)) + bytes(C.c_uint64(m.density_grid or 0)) + bytes(C.c_float(m.grid_max_density)))


def _box(b):
    return bytes(b.lo) + bytes(b.hi)


@pytest.mark.parametrize("sun", [1, 0])
def test_cloud_scene_matches_reference(sun):
    """mc_scene_cloud against the reference's own setup_scene(Cloud)
    (buildCloudScene and the grid-material loop, then finalizeScene), run from
    oracle/_ref with the same grid bounds, maximum and grid pointer (only
    stored, never read): every triangle and sphere field equal, and main()'s
    cloud film and camera settings."""
    import mcref
    h = mcpt.VolumeGrid()
    wmin, wmax = (-120.5, 10.25, -80.0), (130.75, 190.5, 60.125)
    for a in range(3):
        h.world_min[a], h.world_max[a] = wmin[a], wmax[a]
    h.maximum_density = 0.873
    grid = 0x7F00  # a stand-in device pointer: the scene only carries it
    s = mcpt.SceneHost()
    mcpt.check(mcpt.load().mc_scene_cloud(grid, C.byref(h), sun, C.byref(s)))
    tris = (mcpt.Triangle * 8)()
    sph = (mcpt.Sphere * 4)()
    nt, ns = C.c_int32(), C.c_int32()
    rc = mcref.load(False).mcref_cloud_scene((C.c_float * 3)(*wmin), (C.c_float * 3)(*wmax), 0.873, grid, sun,
                                             C.addressof(tris), 8, C.byref(nt), C.addressof(sph), 4, C.byref(ns))
    assert rc == 0 and (s.triangle_count, s.sphere_count) == (nt.value, ns.value) == (4 if sun else 2, 1)
    mine_t, mine_s = mcpt.host_triangles(s), mcpt.host_spheres(s)
    for i in range(nt.value):
        assert bytes(mine_t[i])[:96] == bytes(tris[i])[:96]
        assert _mat(mine_t[i].mat) == _mat(tris[i].mat) and _box(mine_t[i].aabb) == _box(tris[i].aabb)
    a, b = mine_s[0], sph[0]
    assert bytes(a.center) + bytes(a.center1) + bytes(C.c_float(a.radius)) == \
        bytes(b.center) + bytes(b.center1) + bytes(C.c_float(b.radius))
    assert a.is_moving == b.is_moving and _mat(a.mat) == _mat(b.mat) and _box(a.aabb) == _box(b.aabb)
    assert a.mat.density_grid == grid and a.mat.grid_max_density == np.float32(0.873)
    # main()'s cloud settings (PT:4080-4084, 4148-4167)
    f32 = np.float32
    hfov = f32(54.43) * f32(np.pi) / f32(180)
    vfov = f32(2) * np.arctan(np.tan(hfov * f32(0.5)) / (f32(333) / f32(180))) * f32(180) / f32(np.pi)
    assert (s.width, s.height, s.spp, s.max_depth) == (333, 180, 500, 1000)
    assert abs(s.camera.vfov - vfov) <= 1e-5 * vfov
    assert s.camera.rr_cap == f32(0.95) and tuple(s.camera.up.__getattribute__(k) for k in "xyz") == \
        tuple(f32(v) for v in (0.273, 0.962, -0.009))
    assert s.has_medium == mcpt.MEDIUM_ANY | mcpt.MEDIUM_GRID
    mcpt.free_scene(s)


def test_oracle_grid_stand_in_reads_as_the_trilinear_restatement():
    """The oracle's nanovdb stand-in (the grid the reference's trackers read in
    the parity tests), called on the host through the reference's call chain
    (PT:784-789), against a float64 restatement of the trilinear reading:
    index point (p - origin) * (1 / voxel) in float32, 8 voxels around its floor
    (0 outside), along z, then y, then x."""
    import mcref
    rng = np.random.default_rng(2)
    nx, ny, nz = 9, 6, 7
    d = rng.random((nz, ny, nx)).astype(np.float32) * 3
    h = mcpt.VolumeGrid()
    org = np.float32([-0.4, 0.25, 1.0])
    voxel = np.float32(0.13)
    for a in range(3):
        h.origin[a] = org[a]
    h.voxel_size = voxel
    h.inv_voxel_size = np.float32(1) / voxel
    h.dims[0], h.dims[1], h.dims[2] = nx, ny, nz
    h.maximum_density = d.max()
    blob = np.frombuffer(bytes(h) + d.tobytes(), np.uint8).copy()
    pts = rng.uniform(org - 0.3, org + voxel * np.float32([nx, ny, nz]) + 0.3, (20000, 3)).astype(np.float32)
    pts[:200] = org + voxel * rng.integers(-1, 10, (200, 3)).astype(np.float32)
    out = np.zeros(len(pts), np.float32)
    assert mcref.load(False).mcref_grid_sample(blob.ctypes.data, pts.ctypes.data, len(pts), out.ctypes.data) == 0
    x = ((pts - org) * h.inv_voxel_size).astype(np.float64)
    f = np.floor(x)
    i = f.astype(np.int64)
    u = x - f

    def at(a, b, c):
        ok = (a >= 0) & (b >= 0) & (c >= 0) & (a < nx) & (b < ny) & (c < nz)
        v = np.zeros(len(a))
        v[ok] = d[c[ok], b[ok], a[ok]]
        return v

    def lerp(a, b, w):
        return a + w * (b - a)
    ix, iy, iz = i[:, 0], i[:, 1], i[:, 2]
    zs = [lerp(at(ix + a, iy + b, iz), at(ix + a, iy + b, iz + 1), u[:, 2]) for a in (0, 1) for b in (0, 1)]
    want = lerp(lerp(zs[0], zs[1], u[:, 1]), lerp(zs[2], zs[3], u[:, 1]), u[:, 0])
    assert np.abs(out - want).max() <= 1e-6 * 3


def test_cloud_scene_rejects_a_grid_without_extent():
    h = mcpt.VolumeGrid()
    for a in range(3):
        h.world_min[a] = h.world_max[a] = 1.0
    s = mcpt.SceneHost()
    lib = mcpt.load()
    assert lib.mc_scene_cloud(0x7F00, C.byref(h), 1, C.byref(s)) == 1
    assert lib.mc_scene_cloud(None, C.byref(h), 1, C.byref(s)) == 1
