"""CPU tests: the oracle against the golden fixtures made from the reference,
the host logic of the library, the C ABI's exported surface and its error
behaviour without a GPU."""
import ctypes as C
import hashlib
import os
import re

import numpy as np
import pytest

import mcpt
import mcref
from helpers import GOLDEN, ROOT, node_fields, oracle, oracle_build, oracle_sort, primary_rays

# ---------------------------------------------------------------------------
# Philox known-answer tests (Random123 distribution, kat_vectors: philox4x32 10)
# ---------------------------------------------------------------------------
KAT = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
       ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
       ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
        (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]


@pytest.mark.parametrize("ctr,key,expect", KAT)
def test_oracle_philox_known_answers(ctr, key, expect):
    c = np.array(ctr, np.uint32)
    k = np.array(key, np.uint32)
    out = np.zeros(4, np.uint32)
    oracle().orc_philox4x32_10(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    assert tuple(int(x) for x in out) == expect


# ---------------------------------------------------------------------------
# Oracle vs golden fixtures of the reference's host-side code
# ---------------------------------------------------------------------------
def _scene(name):
    kind, variant = {"cornell": (mcpt.SCENE_CORNELL_BOXES, 0), "ico3": (mcpt.SCENE_DISPLACED_ICOSPHERES, 3)}[name]
    return mcpt.generate_scene(kind, variant=variant, seed=2)


@pytest.mark.parametrize("name", ["cornell", "ico3"])
def test_scene_generator_matches_fixture_scene(name):
    g = np.load(os.path.join(GOLDEN, "%s_host.npz" % name))
    s = _scene(name)
    tris = mcpt.host_triangles(s)
    digest = hashlib.sha256(np.frombuffer(tris, dtype=np.uint8).tobytes()).hexdigest()
    assert digest == str(g["scene_sha256"]), "the seeded scene generator changed"
    mcpt.free_scene(s)


@pytest.mark.parametrize("name", ["cornell", "ico3"])
def test_oracle_morton_sort_bounds_match_reference(name):
    g = np.load(os.path.join(GOLDEN, "%s_host.npz" % name))
    s = _scene(name)
    codes, srt, perm, boxes, sb = oracle_sort(mcpt.host_triangles(s))
    assert np.array_equal(codes, g["codes"])
    assert np.array_equal(srt, g["sorted"])
    assert np.array_equal(perm, g["perm"]), "std::sort tie order"
    assert np.array_equal(sb.view(np.uint32)[[0, 1, 2, 4, 5, 6]], g["scene_bounds"].view(np.uint32)[[0, 1, 2, 4, 5, 6]])
    sorted_boxes = boxes[perm]
    gb = g["sorted_bounds"]
    assert np.array_equal(sorted_boxes[:, [0, 1, 2, 4, 5, 6]].view(np.uint32), gb[:, [0, 1, 2, 4, 5, 6]].view(np.uint32))
    mcpt.free_scene(s)


@pytest.mark.parametrize("name", ["cornell", "ico3"])
def test_camera_and_lights_match_reference(name):
    g = np.load(os.path.join(GOLDEN, "%s_host.npz" % name))
    s = _scene(name)
    assert bytes(s.camera) == g["camera"].tobytes(), "Camera::initialize"
    cam = mcpt.Camera.from_buffer_copy(g["camera_input"].tobytes())
    mcpt.camera_initialize(cam)
    assert bytes(cam) == g["camera"].tobytes()
    tris = mcpt.host_triangles(s)
    n = len(tris)
    nl = C.c_int32()
    lights = (mcpt.Light * n)()
    tcopy = (mcpt.Triangle * n)()
    C.memmove(tcopy, tris, C.sizeof(mcpt.Triangle) * n)
    mcpt.check(mcpt.load().mc_scene_finalize_host(C.addressof(tcopy), n, C.addressof(lights), C.byref(nl)))
    got = np.frombuffer(lights, np.float32, count=nl.value * 16).reshape(nl.value, 16)
    assert np.array_equal(got.view(np.uint32), g["lights"].view(np.uint32))
    mcpt.free_scene(s)


def test_full_scene_host_digests():
    """Morton codes and std::sort order on the full 3,932,176-triangle scene."""
    g = np.load(os.path.join(GOLDEN, "full_icospheres_host_digest.npz"))
    s = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=8, seed=2)
    tris = mcpt.host_triangles(s)
    assert hashlib.sha256(np.frombuffer(tris, dtype=np.uint8).tobytes()).hexdigest() == str(g["scene_sha256"])
    codes, srt, perm, boxes, sb = oracle_sort(tris)
    assert hashlib.sha256(codes.tobytes()).hexdigest() == str(g["codes_sha256"])
    assert hashlib.sha256(srt.tobytes()).hexdigest() == str(g["sorted_sha256"])
    assert hashlib.sha256(perm.tobytes()).hexdigest() == str(g["perm_sha256"])
    mcpt.free_scene(s)


def _device_fixture(name):
    p = os.path.join(GOLDEN, "%s_device.npz" % name)
    if not os.path.exists(p):
        pytest.skip("device fixtures not generated yet (tests/golden/make_golden.py --gpu)")
    return np.load(p)


@pytest.mark.parametrize("name", ["cornell", "ico3"])
def test_oracle_topology_matches_reference_device_build(name):
    d = _device_fixture(name)
    s = _scene(name)
    tris = mcpt.host_triangles(s)
    n = len(tris)
    codes, srt, perm, boxes, sb = oracle_sort(tris)
    internal, leaves = oracle_build(srt, perm, boxes)
    mi = node_fields(bytes(internal), n - 1)
    ri = node_fields(d["internal"].tobytes(), n - 1)
    for nm, a, b in zip(["bounds", "left", "right", "lleaf", "rleaf", "parent"], mi[:6], ri[:6]):
        if nm == "bounds":
            assert np.array_equal(a[:, [0, 1, 2, 4, 5, 6]].view(np.uint32), b[:, [0, 1, 2, 4, 5, 6]].view(np.uint32))
        else:
            assert np.array_equal(a, b), nm
    ml = node_fields(bytes(leaves), n)
    rl = node_fields(d["leaves"].tobytes(), n)
    assert np.array_equal(ml[6], rl[6]) and np.array_equal(ml[5], rl[5])
    mcpt.free_scene(s)


@pytest.mark.parametrize("name", ["cornell", "ico3"])
def test_oracle_hits_match_reference_device_hits(name):
    """IEEE CPU arithmetic vs the reference's fast-math GPU arithmetic: ids agree
    except on numerical near-ties, t within 1e-4 relative."""
    d = _device_fixture(name)
    s = _scene(name)
    tris = mcpt.host_triangles(s)
    n = len(tris)
    codes, srt, perm, boxes, sb = oracle_sort(tris)
    internal, leaves = oracle_build(srt, perm, boxes)
    types = np.ones(n, np.int32)
    hot = (mcpt.TriangleHot * n)()
    cold = (mcpt.TriangleCold * n)()
    mcpt.check(mcpt.load().mc_split_triangles_host(C.addressof(tris), n, C.addressof(hot), C.addressof(cold)))
    rays = np.ascontiguousarray(d["rays"])
    nr = rays.shape[1]
    hits = (mcpt.PackedHit * nr)()
    oracle().orc_trace(C.addressof(internal), C.addressof(leaves), types.ctypes.data, n, C.addressof(hot), None,
                       rays.ctypes.data, nr, 0, None, C.addressof(hits), None, 4)
    mine = np.frombuffer(hits, np.int32).reshape(nr, 4)
    ref = d["hits"]
    same = mine[:, 2] == ref[:, 2]
    assert same.mean() > 0.998
    both = (mine[:, 3] == 1) & (ref[:, 3] == 1)
    tm = mine[both, 0].view(np.float32)
    tr = ref[both, 0].view(np.float32)
    assert np.all(np.abs(tm - tr) <= 1e-4 * np.abs(tr) + 1e-6)
    occ = np.zeros(nr, np.int32)
    tmax = np.ascontiguousarray(d["tmax"])
    oracle().orc_trace(C.addressof(internal), C.addressof(leaves), types.ctypes.data, n, C.addressof(hot), None,
                       rays.ctypes.data, nr, 1, tmax.ctypes.data, None, occ.ctypes.data, 4)
    assert (occ == d["occluded"]).mean() > 0.998
    mcpt.free_scene(s)


@pytest.mark.parametrize("name", ["cornell", "ico3"])
def test_oracle_image_matches_reference_device_image(name):
    """Same counter-based draws; per-pixel agreement of the FP32 oracle with the
    reference's fast-math image, and the images' means within 1%."""
    d = _device_fixture(name)
    s = _scene(name)
    tris = mcpt.host_triangles(s)
    env = mcpt.host_env(s)
    orc = oracle()
    h = orc.orc_scene_create(C.addressof(tris), len(tris), None, 0, env.ctypes.data if env is not None else None,
                             s.env_width, s.env_height, s.env_intensity, 0.0)
    ref = d["image"]
    H, W = ref.shape[:2]
    spp = int(d["image_spp"])
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = W / float(H)
    mcpt.camera_initialize(cam)
    acc = np.zeros(W * H * 3, np.float64)
    stats = np.zeros(2, np.float64)
    orc.orc_render(h, C.addressof(cam), W, H, spp, 0, 8, 1234, 0, 0, 0, 0, W, H, os.cpu_count() or 1, acc.ctypes.data,
                   stats.ctypes.data)
    orc.orc_scene_destroy(h)
    img = acc.reshape(H, W, 3)
    close = np.all(np.abs(img - ref) <= 1e-3 * np.maximum(np.abs(ref), 1e-2), axis=2).mean()
    assert close > 0.9, close
    assert abs(img.mean() - ref.mean()) <= 0.01 * ref.mean()
    assert abs(stats[0] - d["image_rays"][0]) <= 0.02 * d["image_rays"][0]
    mcpt.free_scene(s)


def test_oracle_fp32_and_fp64_estimators_agree():
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
    tris = mcpt.host_triangles(s)
    orc = oracle()
    h = orc.orc_scene_create(C.addressof(tris), len(tris), None, 0, None, 0, 0, 1.0, 0.0)
    W = H = 24
    cam = mcpt.make_camera(W, H, (0, 2, 5.5), (0, 2, -2), 40.0, 7.5)
    out = []
    for dbl in (0, 1):
        acc = np.zeros(W * H * 3, np.float64)
        orc.orc_render(h, C.addressof(cam), W, H, 64, 0, 8, 77, dbl, 0, 0, 0, W, H, 4, acc.ctypes.data, None)
        out.append(acc.reshape(H, W, 3) / 64)
    orc.orc_scene_destroy(h)
    assert abs(out[0].mean() - out[1].mean()) < 0.01 * out[1].mean()
    mcpt.free_scene(s)


# ---------------------------------------------------------------------------
# The reference build itself (host side runs without a GPU) when it is present
# ---------------------------------------------------------------------------
@pytest.mark.skipif(not mcref.available(False), reason="oracle/_ref not built (needs the reference sources)")
def test_reference_host_outputs_match_fixtures():
    g = np.load(os.path.join(GOLDEN, "ico3_host.npz"))
    s = _scene("ico3")
    tris = mcpt.host_triangles(s)
    n = len(tris)
    out = {k: np.zeros(n, np.uint32 if k in ("codes", "sorted") else np.int32) for k in ("codes", "sorted", "ids", "types", "perm")}
    sb = np.zeros(n * 8, np.float32)
    bb = np.zeros(8, np.float32)
    tb = np.zeros(n * 8, np.float32)
    lights = np.zeros(n * 16, np.float32)
    nl = C.c_int32()
    assert mcref.load(False).mcref_finalize_and_sort(C.addressof(tris), n, None, 0, out["codes"].ctypes.data,
                                                     out["sorted"].ctypes.data, out["ids"].ctypes.data,
                                                     out["types"].ctypes.data, out["perm"].ctypes.data, sb.ctypes.data,
                                                     bb.ctypes.data, tb.ctypes.data, lights.ctypes.data, C.byref(nl)) == 0
    for k in ("codes", "sorted", "perm", "ids"):
        assert np.array_equal(out[k], g[k])
    mcpt.free_scene(s)


# ---------------------------------------------------------------------------
# The C ABI: every declared symbol is exported; failures come back as statuses
# ---------------------------------------------------------------------------
def declared_functions():
    src = open(os.path.join(ROOT, "include", "mc_abi.h")).read()
    return sorted(set(re.findall(r"MC_API\s+[A-Za-z_][A-Za-z0-9_ \*]*?\b(mc_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = mcpt.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = os.popen("nm -D --defined-only %s" % mcpt.LIB_PATH).read()
    exported = set(re.findall(r" T (mc_[a-z0-9_]+)", out))
    assert set(names) <= exported
    assert all(n in mcpt.SIGNATURES for n in names), "binding misses a declared function"


def test_errors_are_statuses_not_exits():
    lib = mcpt.load()
    h = C.c_void_p()
    st = lib.mc_context_create(0, C.byref(h))
    if st == 0:
        lib.mc_context_destroy(h)
        pytest.skip("a GPU is present")
    assert st == 10  # MC_ERR_UNSUPPORTED without a device
    assert b"no CUDA device" in lib.mc_last_error()
    assert lib.mc_camera_initialize(None) == 1
    assert lib.mc_scene_generate(None, None) == 1
    d = mcpt.SceneDesc(99, 0, 0, 0)
    s = mcpt.SceneHost()
    assert lib.mc_scene_generate(C.byref(d), C.byref(s)) == 1
    assert lib.mc_bvh_build(None, None, None, None) == 1
    assert lib.mc_status_string(4) == b"traversal stack overflow"


def test_scene_generators_are_deterministic_and_sized():
    a = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
    assert a.triangle_count == 36 and (a.width, a.height, a.spp, a.max_depth) == (512, 512, 64, 8)
    b = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=2, seed=2)
    c = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=2, seed=2)
    assert b.triangle_count == 3 * 20 * 16 + 16
    assert bytes(mcpt.host_triangles(b)) == bytes(mcpt.host_triangles(c))
    assert b.has_medium == 1 and b.env_width == 2048 and b.env_height == 1024
    env = mcpt.host_env(b)
    assert env.shape == (1024, 2048, 4) and float(env[..., :3].max()) > 400  # the sun
    for member in (0, 1, 17):
        m = mcpt.generate_scene(mcpt.SCENE_BATCH_MEMBER, variant=member, seed=3, triangle_target=2000)
        assert 1000 <= m.triangle_count <= 4000
        assert m.width in (256, 512, 1024) and m.spp in (4, 16, 64)
        mcpt.free_scene(m)
    r = mcpt.generate_scene(mcpt.SCENE_GUIDING_ROOM, seed=4)
    assert 150000 <= r.triangle_count <= 250000 and (r.width, r.height) == (1024, 1024)
    for s in (a, b, c, r):
        mcpt.free_scene(s)


@pytest.mark.skipif(not mcref.available(False), reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("kind,variant,seed", [(mcpt.SCENE_CORNELL_BOXES, 0, 0), (mcpt.SCENE_DISPLACED_ICOSPHERES, 5, 2),
                                               (mcpt.SCENE_BATCH_MEMBER, 3, 3), (mcpt.SCENE_GUIDING_ROOM, 0, 4),
                                               (mcpt.SCENE_CORNELL_SPHERES, 0, 2)])
def test_reference_harness_generates_the_library_scenes(kind, variant, seed):
    """The benchmark's reference arm reads its scene through the harness's copy
    of the generator (no library loaded there): the same bytes as the library's."""
    a = mcpt.generate_scene(kind, variant=variant, seed=seed)
    b = mcref.SceneHost()
    assert mcref.load(False).mcref_generate_scene(kind, variant, seed, 0, C.byref(b)) == 0
    try:
        assert b.triangle_count == a.triangle_count and b.sphere_count == a.sphere_count
        assert C.string_at(b.triangles, 224 * b.triangle_count) == bytes(mcpt.host_triangles(a))
        if a.sphere_count:
            assert C.string_at(b.spheres, 160 * b.sphere_count) == C.string_at(a.spheres, 160 * a.sphere_count)
        assert bytes(b.camera) == bytes(a.camera)
        assert (b.width, b.height, b.spp, b.max_depth, b.has_medium) == (a.width, a.height, a.spp, a.max_depth,
                                                                         a.has_medium)
        assert (b.env_width, b.env_height, b.env_intensity) == (a.env_width, a.env_height, a.env_intensity)
        if a.env_width:
            nb = 16 * a.env_width * a.env_height
            assert C.string_at(b.env_rgba, nb) == C.string_at(C.cast(a.env_rgba, C.c_void_p), nb)
    finally:
        mcref.load(False).mcref_free_scene(C.byref(b))
        mcpt.free_scene(a)


def test_primary_rays_helper_matches_camera():
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
    r = primary_rays(s.camera, 8, 8)
    assert r.shape == (7, 64)
    assert np.allclose(np.linalg.norm(r[3:6], axis=0), 1.0, atol=1e-6)
    mcpt.free_scene(s)


def test_host_finalize_matches_reference_on_random_soup():
    """mc_scene_finalize_host against the reference's finalizeScene on 5,000
    random triangles, 30 % emissive: bounds and the light list bit-exact."""
    rng = np.random.default_rng(11)
    s = _scene("ico3")
    src = np.frombuffer(mcpt.host_triangles(s), np.uint8).reshape(-1, 224)
    n = 5000
    a = src[rng.integers(0, len(src), n)].copy()
    a[:, 0:36] = rng.uniform(-1, 1, (n, 9)).astype(np.float32).view(np.uint8)
    a[:, 96:100] = np.where(rng.random(n) < 0.3, mcpt.MAT_EMISSIVE, 0).astype(np.int32).view(np.uint8).reshape(n, 4)
    mcpt.free_scene(s)
    tris = (mcpt.Triangle * n)()
    C.memmove(tris, a.ctypes.data, n * 224)
    tb = np.zeros(n * 8, np.float32)
    rl = np.zeros(n * 16, np.float32)
    rn = C.c_int32()
    assert mcref.load(False).mcref_finalize_and_sort(C.addressof(tris), n, None, 0, None, None, None, None, None, None,
                                                     None, tb.ctypes.data, rl.ctypes.data, C.byref(rn)) == 0
    hl = (mcpt.Light * n)()
    hn = C.c_int32()
    mcpt.check(mcpt.load().mc_scene_finalize_host(C.addressof(tris), n, C.addressof(hl), C.byref(hn)))
    assert hn.value == rn.value > 1000
    assert np.frombuffer(hl, np.uint8)[:hn.value * 64].tobytes() == rl.view(np.uint8)[:rn.value * 64].tobytes()
    boxes = np.frombuffer(tris, np.uint8).reshape(n, 224)[:, 192:224].copy().view(np.float32)
    lanes = [0, 1, 2, 4, 5, 6]
    assert np.array_equal(boxes[:, lanes].view(np.uint32), tb.reshape(n, 8)[:, lanes].view(np.uint32))


def _png_pixels(png):
    """Decodes a PNG of 8-bit RGB with filter type 0 rows: checks the chunk
    CRCs and returns (width, height, pixels)."""
    import struct
    import zlib
    assert png[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, ihdr = 8, b"", None
    while pos < len(png):
        (length,) = struct.unpack(">I", png[pos:pos + 4])
        ctype, data = png[pos + 4:pos + 8], png[pos + 8:pos + 8 + length]
        (crc,) = struct.unpack(">I", png[pos + 8 + length:pos + 12 + length])
        assert crc == zlib.crc32(ctype + data) & 0xFFFFFFFF, ctype
        if ctype == b"IHDR":
            ihdr = struct.unpack(">IIBBBBB", data)
        elif ctype == b"IDAT":
            idat += data
        pos += 12 + length
        if ctype == b"IEND":
            break
    assert pos == len(png)
    w, h, depth, colour, comp, filt, interlace = ihdr
    assert (depth, colour, comp, filt, interlace) == (8, 2, 0, 0, 0)
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)
    assert (raw[:, 0] == 0).all()
    return w, h, raw[:, 1:].reshape(h, w, 3)


@pytest.mark.parametrize("w,h", [(1, 1), (37, 23), (300, 250), (1920, 12)])
def test_png_encoder_round_trip(w, h):
    """mc_png_encode: valid chunks and CRCs, a zlib stream (stored blocks,
    more than one once a row set passes 65,535 bytes) that decodes to the
    same pixels."""
    rng = np.random.default_rng(w * 1000 + h)
    px = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    png = mcpt.png_encode(px, w, h)
    gw, gh, got = _png_pixels(png)
    assert (gw, gh) == (w, h)
    assert np.array_equal(got, px)


def test_png_encoder_rejects_bad_sizes():
    n = C.c_int64(0)
    assert mcpt.load().mc_png_encode(None, 0, 5, None, C.byref(n)) == 1
    assert mcpt.load().mc_png_encode(None, 4, 4, None, None) == 1
    n = C.c_int64(10)
    buf = (C.c_uint8 * 10)()
    px = np.zeros(48, np.uint8)
    assert mcpt.load().mc_png_encode(px.ctypes.data, 4, 4, buf, C.byref(n)) == 1
