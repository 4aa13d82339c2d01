"""Density grids on the host (no GPU): the fog sphere of
createFogSphereGrid (src/volume_io.cpp:53-64) as mc_volume_fog_sphere builds
it, the grid header's layout, and argument checks."""
import ctypes as C

import numpy as np

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
