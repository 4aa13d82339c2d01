"""Scene ingestion on the device (mc_scene_ingest): triangle bounds and the
light list of the reference's finalizeScene (PT:1930-1987) and the hot/cold
split of its main() (PT:4276-4289).

Bars: bit-exact. Bounds and lights against the reference's own finalizeScene
(oracle/_ref, host code), hot and cold records byte for byte against the host
split, on the seeded scenes, the full 3,932,176-triangle scene, random triangle
soups with ragged sizes (1, 127, 128, 129, ...) and many lights spread over
thousands of tiles, and a scene with no triangles.
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


def ingest(ctx, tris, spheres=None, via_host=False, src_ptr=None):
    """Runs mc_scene_ingest on a device copy of a host triangle array (or
    mc_scene_ingest_host on the host array itself, or on src_ptr); returns
    numpy views of hot (n, 36), cold (n, 192), lights (count, 64) bytes and
    has_medium."""
    n = len(tris)
    ns = len(spheres) if spheres is not None else 0
    aos = torch.frombuffer(tris, dtype=torch.uint8, count=n * 224).cuda() if n and not via_host else None
    sph = torch.frombuffer(spheres, dtype=torch.uint8, count=ns * 160).cuda() if ns else None
    hot = torch.full((max(n, 1) * 36,), 0xAB, dtype=torch.uint8, device="cuda")
    cold = torch.full((max(n, 1) * 192,), 0xAB, dtype=torch.uint8, device="cuda")
    lights = torch.full((max(n, 1) * 64,), 0xAB, dtype=torch.uint8, device="cuda")
    nl, med = C.c_int32(-1), C.c_int32(-1)
    torch.cuda.synchronize()
    if via_host:
        src = src_ptr if src_ptr is not None else (C.addressof(tris) if n else None)
        mcpt.check(mcpt.load().mc_scene_ingest_host(ctx.handle, src, n, sph.data_ptr() if ns else None, ns,
                                                    hot.data_ptr(), cold.data_ptr(), lights.data_ptr(), C.byref(nl),
                                                    C.byref(med)))
    else:
        mcpt.check(mcpt.load().mc_scene_ingest(ctx.handle, aos.data_ptr() if n else None, n,
                                               sph.data_ptr() if ns else None, ns, hot.data_ptr(), cold.data_ptr(),
                                               lights.data_ptr(), C.byref(nl), C.byref(med)))
    return (hot.cpu().numpy()[:n * 36].reshape(n, 36), cold.cpu().numpy()[:n * 192].reshape(n, 192),
            lights.cpu().numpy()[:nl.value * 64].reshape(nl.value, 64), med.value)


def host_split(tris):
    n = len(tris)
    hot = (mcpt.TriangleHot * max(n, 1))()
    cold = (mcpt.TriangleCold * max(n, 1))()
    tcopy = (mcpt.Triangle * max(n, 1))()
    C.memmove(tcopy, tris, C.sizeof(mcpt.Triangle) * n)
    mcpt.check(mcpt.load().mc_scene_finalize_host(C.addressof(tcopy), n, None, None))
    mcpt.check(mcpt.load().mc_split_triangles_host(C.addressof(tcopy), n, C.addressof(hot), C.addressof(cold)))
    return (np.frombuffer(hot, np.uint8, count=n * 36).reshape(n, 36),
            np.frombuffer(cold, np.uint8, count=n * 192).reshape(n, 192))


def reference_finalize(tris, spheres=None):
    """Triangle bounds (n, 8) f32 and the light list (count, 64) bytes from the
    reference's finalizeScene."""
    n = len(tris)
    ns = len(spheres) if spheres is not None else 0
    tb = np.zeros(max(n, 1) * 8, np.float32)
    lights = np.zeros(max(n, 1) * 16, np.float32)
    nl = C.c_int32()
    assert mcref.load(False).mcref_finalize_and_sort(C.addressof(tris), n, C.addressof(spheres) if ns else None, ns,
                                                     None, None, None, None, None, None, None, tb.ctypes.data,
                                                     lights.ctypes.data, C.byref(nl)) == 0
    return tb[:n * 8].reshape(n, 8), lights.view(np.uint8)[:nl.value * 64].reshape(nl.value, 64)


def check_against_reference(ctx, tris, spheres=None, expect_medium=None, via_host=False):
    hot, cold, lights, med = ingest(ctx, tris, spheres, via_host=via_host)
    h_hot, h_cold = host_split(tris)
    assert np.array_equal(hot, h_hot), "hot records differ from the host split"
    assert np.array_equal(cold, h_cold), "cold records differ from the host split"
    tb, ref_lights = reference_finalize(tris, spheres)
    boxes = cold[:, 160:192].copy().view(np.float32)
    lanes = [0, 1, 2, 4, 5, 6]
    assert np.array_equal(boxes[:, lanes].view(np.uint32), tb[:, lanes].view(np.uint32)), "bounds differ from finalizeScene"
    assert lights.shape == ref_lights.shape, "light count differs from finalizeScene"
    assert np.array_equal(lights, ref_lights), "lights differ from finalizeScene"
    if expect_medium is not None:
        assert med == int(expect_medium)
    return lights.shape[0]


@pytest.mark.parametrize("kind,variant", [(mcpt.SCENE_CORNELL_BOXES, 0), (mcpt.SCENE_DISPLACED_ICOSPHERES, 3),
                                          (mcpt.SCENE_CORNELL_SPHERES, 0)])
def test_ingest_matches_reference_finalize_and_host_split(ctx, kind, variant):
    s = mcpt.generate_scene(kind, variant=variant, seed=2)
    tris = mcpt.host_triangles(s)
    sph = mcpt.host_spheres(s)
    types = [tris[i].mat.type for i in range(len(tris))] + ([sph[i].mat.type for i in range(len(sph))] if sph else [])
    nl = check_against_reference(ctx, tris, sph, expect_medium=mcpt.MAT_ISOTROPIC in types)
    assert nl >= 1
    mcpt.free_scene(s)


def soup(n, seed, emissive_frac=0.1, medium_frac=0.0):
    """n random triangles: vertices ~U[-1,1]^3, random uv/normal bytes, garbage
    input boxes, material records taken from a generated scene (their padding
    as the generator writes it) with random types."""
    rng = np.random.default_rng(seed)
    s = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=1, seed=seed)
    src = np.frombuffer(mcpt.host_triangles(s), np.uint8).reshape(-1, 224)
    a = src[rng.integers(0, len(src), n)].copy()
    a[:, 0:36] = rng.uniform(-1, 1, (n, 9)).astype(np.float32).view(np.uint8)
    a[:, 36:96] = rng.uniform(-1, 1, (n, 15)).astype(np.float32).view(np.uint8)
    a[:, 192:224] = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    types = np.where(rng.random(n) < emissive_frac, mcpt.MAT_EMISSIVE,
                     np.where(rng.random(n) < medium_frac, mcpt.MAT_ISOTROPIC, 0)).astype(np.int32)
    a[:, 96:100] = types.view(np.uint8).reshape(n, 4)
    mcpt.free_scene(s)
    arr = (mcpt.Triangle * n)()
    C.memmove(arr, a.ctypes.data, n * 224)
    return arr, types


@pytest.mark.parametrize("n", [1, 127, 128, 129, 1000, 4097])
@pytest.mark.parametrize("via_host", [False, True])
def test_ingest_ragged_sizes(ctx, n, via_host):
    tris, types = soup(n, seed=n, emissive_frac=0.3)
    nl = check_against_reference(ctx, tris, expect_medium=False, via_host=via_host)
    assert nl == int((types == mcpt.MAT_EMISSIVE).sum())


@pytest.mark.parametrize("via_host", [False, True])
def test_ingest_many_lights_over_many_tiles(ctx, via_host):
    """300,000 triangles = 2,344 tiles (the offset scan runs three rounds),
    about 10 % emissive, spread over every tile; a few isotropic ones. From a
    host array of 67 MB the upload goes through the pinned staging threads."""
    tris, types = soup(300000, seed=7, emissive_frac=0.1, medium_frac=0.001)
    nl = check_against_reference(ctx, tris, expect_medium=True, via_host=via_host)
    assert nl == int((types == mcpt.MAT_EMISSIVE).sum()) > 25000


def test_ingest_host_from_pinned_memory(ctx):
    """A pinned host array is copied directly (no staging); same bytes."""
    tris, types = soup(200000, seed=9, emissive_frac=0.05)
    pinned = torch.empty(len(tris) * 224, dtype=torch.uint8, pin_memory=True)
    pinned.copy_(torch.frombuffer(tris, dtype=torch.uint8, count=len(tris) * 224))
    a = ingest(ctx, tris)
    b = ingest(ctx, tris, via_host=True, src_ptr=pinned.data_ptr())
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert a[3] == b[3]


def test_ingest_no_triangles_spheres_only(ctx):
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_SPHERES, seed=2)
    sph = mcpt.host_spheres(s)
    assert sph is not None
    hot, cold, lights, med = ingest(ctx, (mcpt.Triangle * 0)(), sph)
    assert lights.shape[0] == 0
    assert med == int(any(sph[i].mat.type == mcpt.MAT_ISOTROPIC for i in range(len(sph))))
    mcpt.free_scene(s)


def test_ingest_full_scene(ctx):
    s = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=8, seed=2)
    tris = mcpt.host_triangles(s)
    assert len(tris) == 3932176
    hot, cold, lights, med = ingest(ctx, tris)
    h_hot, h_cold = host_split(tris)
    assert np.array_equal(hot, h_hot) and np.array_equal(cold, h_cold)
    via = ingest(ctx, tris, via_host=True)
    assert all(np.array_equal(x, y) for x, y in zip((hot, cold, lights), via[:3])) and via[3] == med
    tcopy = (mcpt.Triangle * len(tris))()
    C.memmove(tcopy, tris, C.sizeof(mcpt.Triangle) * len(tris))
    nl = C.c_int32()
    mcpt.check(mcpt.load().mc_scene_finalize_host(C.addressof(tcopy), len(tris), None, C.byref(nl)))
    hl = (mcpt.Light * nl.value)()
    mcpt.check(mcpt.load().mc_scene_finalize_host(C.addressof(tcopy), len(tris), C.addressof(hl), C.byref(nl)))
    assert np.array_equal(lights, np.frombuffer(hl, np.uint8).reshape(nl.value, 64))
    assert med == 1
    mcpt.free_scene(s)


def test_ingest_rejects_unaligned_arrays(ctx):
    buf = torch.zeros(224 * 4 + 16, dtype=torch.uint8, device="cuda")
    hot = torch.zeros(36 * 4 + 16, dtype=torch.uint8, device="cuda")
    cold = torch.zeros(192 * 4 + 16, dtype=torch.uint8, device="cuda")
    st = mcpt.load().mc_scene_ingest(ctx.handle, buf.data_ptr() + 4, 4, None, 0, hot.data_ptr(), cold.data_ptr(),
                                     None, None, None)
    assert mcpt.STATUS_NAMES[st] == "MC_ERR_INVALID"


def test_render_from_device_ingest_equals_host_upload(ctx):
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES, seed=2)
    tris = mcpt.host_triangles(s)
    images = []
    for c in (None, ctx):
        ds = mcpt.DeviceScene(tris, ctx=c)
        bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4)
        acc = torch.zeros(64 * 64 * 3, dtype=torch.float32, device="cuda")
        p = mcpt.render_params(s.camera, 64, 64, 4, 8)
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               None))
        torch.cuda.synchronize()
        images.append(acc.cpu().numpy())
        bvh.close()
    assert np.array_equal(images[0], images[1])
    mcpt.free_scene(s)
