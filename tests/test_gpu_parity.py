"""Parity of the CUDA path (through the C ABI) with the UNMODIFIED reference,
compiled in oracle/_ref and run on the same GPU, on the same inputs.

Bars: Morton codes, sorted order and topology bit-exact;
closest-hit ids bit-exact and t within 2 ulp; images per pixel within 1e-4
relative under the same counter-based RNG.
"""
import ctypes as C

import numpy as np
import pytest

import mcpt
import mcref
from helpers import node_fields, primary_rays, random_rays, ulp_diff

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = mcpt.Context(0)
    yield c
    c.close()


_scenes = {}


def scene(kind, variant=0, seed=2):
    key = (kind, variant, seed)
    if key not in _scenes:
        _scenes[key] = mcpt.generate_scene(kind, variant=variant, seed=seed)
    return _scenes[key]


def ref_sort(tris):
    ref = mcref.load()
    n = len(tris)
    a = {k: np.zeros(n, np.uint32 if k in ("codes", "sorted") else np.int32)
         for k in ("codes", "sorted", "ids", "types", "perm")}
    sb = np.zeros(n * 8, np.float32)
    bb = np.zeros(8, np.float32)
    tb = np.zeros(n * 8, np.float32)
    lights = np.zeros(max(n, 1) * 16, np.float32)
    nl = C.c_int32()
    assert ref.mcref_finalize_and_sort(C.addressof(tris), n, None, 0, a["codes"].ctypes.data, a["sorted"].ctypes.data,
                                       a["ids"].ctypes.data, a["types"].ctypes.data, a["perm"].ctypes.data,
                                       sb.ctypes.data, bb.ctypes.data, tb.ctypes.data, lights.ctypes.data,
                                       C.byref(nl)) == 0
    a["sorted_bounds"] = sb.reshape(n, 8)
    a["scene_bounds"] = bb
    return a


def dev(arr):
    return torch.from_numpy(np.ascontiguousarray(arr)).cuda()


CASES = [(mcpt.SCENE_CORNELL_BOXES, 0), (mcpt.SCENE_DISPLACED_ICOSPHERES, 5)]


@pytest.mark.parametrize("kind,variant", CASES + [(mcpt.SCENE_DISPLACED_ICOSPHERES, 8)])
def test_morton_codes_bit_exact(ctx, kind, variant):
    s = scene(kind, variant)
    tris = mcpt.host_triangles(s)
    r = ref_sort(tris)
    ds = mcpt.DeviceScene(tris)
    codes = torch.zeros(len(tris), dtype=torch.int32, device="cuda")
    bounds = mcpt.AABB()
    mcpt.check(ctx.lib.mc_morton_codes(ctx.handle, C.byref(ds.view), codes.data_ptr(), C.byref(bounds)))
    got = codes.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, r["codes"])
    sb = np.array([bounds.lo.x, bounds.lo.y, bounds.lo.z, 0, bounds.hi.x, bounds.hi.y, bounds.hi.z, 0], np.float32)
    assert np.array_equal(sb[[0, 1, 2, 4, 5, 6]], r["scene_bounds"][[0, 1, 2, 4, 5, 6]])


@pytest.mark.parametrize("n,bits", [(1, 30), (7, 30), (5000, 30), (1 << 20, 30), (3932176, 30), (100000, 32)])
def test_radix_sort_stable(ctx, n, bits):
    g = np.random.default_rng(n)
    keys = g.integers(0, 1 << min(bits, 31), n, dtype=np.int64).astype(np.uint32)
    if n > 10:
        keys[: n // 3] = keys[0]  # long run of equal keys
    vals = np.arange(n, dtype=np.int32)
    k = dev(keys.view(np.int32))
    v = dev(vals)
    mcpt.check(ctx.lib.mc_radix_sort_pairs(ctx.handle, k.data_ptr(), v.data_ptr(), n, bits))
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k.cpu().numpy().view(np.uint32), keys[order])
    assert np.array_equal(v.cpu().numpy(), vals[order])


def build_pair(ctx, tris, inject=True):
    r = ref_sort(tris)
    ds = mcpt.DeviceScene(tris)
    perm = dev(r["perm"]) if inject else None
    bvh = mcpt.Bvh(ctx, ds.view, permutation=perm, keep_reference_nodes=True)
    return r, ds, bvh


@pytest.mark.parametrize("kind,variant", CASES + [(mcpt.SCENE_DISPLACED_ICOSPHERES, 8)])
def test_topology_and_bounds_bit_exact(ctx, kind, variant):
    s = scene(kind, variant)
    tris = mcpt.host_triangles(s)
    n = len(tris)
    r, ds, bvh = build_pair(ctx, tris, inject=True)
    ref_int = (mcpt.BvhNode * (n - 1))()
    ref_leaf = (mcpt.BvhNode * n)()
    assert mcref.load().mcref_build_bvh(r["sorted"].ctypes.data, r["ids"].ctypes.data, r["types"].ctypes.data,
                                        r["sorted_bounds"].ctypes.data, n, C.addressof(ref_int), C.addressof(ref_leaf)) == 0
    my_int = torch.zeros((n - 1) * 64, dtype=torch.uint8, device="cuda")
    my_leaf = torch.zeros(n * 64, dtype=torch.uint8, device="cuda")
    codes = torch.zeros(n, dtype=torch.int32, device="cuda")
    bvh.export(codes=codes, internal=my_int, leaves=my_leaf)
    assert np.array_equal(codes.cpu().numpy().view(np.uint32), r["sorted"])
    mi = node_fields(my_int.cpu().numpy().tobytes(), n - 1)
    ri = node_fields(bytes(ref_int), n - 1)
    for name, a, b in zip(["bounds", "left", "right", "lleaf", "rleaf", "parent"], mi[:6], ri[:6]):
        if name == "bounds":
            a, b = a[:, [0, 1, 2, 4, 5, 6]], b[:, [0, 1, 2, 4, 5, 6]]
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
        else:
            assert np.array_equal(a, b), name
    ml = node_fields(my_leaf.cpu().numpy().tobytes(), n)
    rl = node_fields(bytes(ref_leaf), n)
    assert np.array_equal(ml[6], rl[6]), "leaf primitive ids"
    assert np.array_equal(ml[5], rl[5]), "leaf parents"
    assert np.array_equal(ml[0][:, [0, 1, 2, 4, 5, 6]].view(np.uint32), rl[0][:, [0, 1, 2, 4, 5, 6]].view(np.uint32))
    info = bvh.info()
    assert info.primitive_count == n and info.depth <= 64


def test_topology_with_own_stable_order(ctx):
    """Without injecting the reference's std::sort order the sorted codes and the
    tree topology are still identical (they depend only on the code sequence);
    leaf ids differ only inside runs of equal codes."""
    s = scene(mcpt.SCENE_DISPLACED_ICOSPHERES, 5)
    tris = mcpt.host_triangles(s)
    n = len(tris)
    r, ds, bvh = build_pair(ctx, tris, inject=False)
    my_int = torch.zeros((n - 1) * 64, dtype=torch.uint8, device="cuda")
    my_leaf = torch.zeros(n * 64, dtype=torch.uint8, device="cuda")
    codes = torch.zeros(n, dtype=torch.int32, device="cuda")
    bvh.export(codes=codes, internal=my_int, leaves=my_leaf)
    assert np.array_equal(codes.cpu().numpy().view(np.uint32), r["sorted"])
    ref_int = (mcpt.BvhNode * (n - 1))()
    ref_leaf = (mcpt.BvhNode * n)()
    mcref.load().mcref_build_bvh(r["sorted"].ctypes.data, r["ids"].ctypes.data, r["types"].ctypes.data,
                                 r["sorted_bounds"].ctypes.data, n, C.addressof(ref_int), C.addressof(ref_leaf))
    mi = node_fields(my_int.cpu().numpy().tobytes(), n - 1)
    ri = node_fields(bytes(ref_int), n - 1)
    for a, b in zip(mi[1:6], ri[1:6]):
        assert np.array_equal(a, b)
    my_ids = node_fields(my_leaf.cpu().numpy().tobytes(), n)[6]
    # same multiset of ids inside every run of equal codes
    srt = r["sorted"]
    starts = np.flatnonzero(np.r_[True, srt[1:] != srt[:-1]])
    ends = np.r_[starts[1:], n]
    for a, b in zip(starts, ends):
        if b - a > 1:
            assert sorted(my_ids[a:b]) == sorted(r["ids"][a:b])
        else:
            assert my_ids[a] == r["ids"][a]


def upload_ref(s, env=False):
    tris = mcpt.host_triangles(s)
    e = mcpt.host_env(s) if env else None
    ref = mcref.load()
    assert ref.mcref_scene_upload(C.addressof(tris), len(tris), None, 0,
                                  e.ctypes.data if e is not None else None,
                                  s.env_width if e is not None else 0, s.env_height if e is not None else 0,
                                  s.env_intensity, 0.0) == 0
    return ref


@pytest.mark.parametrize("kind,variant", CASES)
@pytest.mark.parametrize("mode", [0, 1])
def test_closest_hits_bit_exact(ctx, kind, variant, mode):
    s = scene(kind, variant)
    tris = mcpt.host_triangles(s)
    r, ds, bvh = build_pair(ctx, tris, inject=True)
    ref = upload_ref(s)
    cam = s.camera
    rays = np.concatenate([primary_rays(cam, s.width, s.height, stride=2 if s.width > 600 else 1),
                           random_rays(200000, -1.5, 1.5, seed=7) if kind == 2 else random_rays(200000, (-1.9, 0.1, -3.9), (1.9, 3.9, -0.1), seed=7)],
                          axis=1)
    rays = np.ascontiguousarray(rays)
    n = rays.shape[1]
    ref_hits = np.zeros((n, 4), np.int32)
    assert ref.mcref_trace(rays.ctypes.data, n, mode, None, ref_hits.ctypes.data, None) == 0
    d_rays = dev(rays)
    d_hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    mcpt.check(ctx.lib.mc_trace_closest(ctx.handle, bvh.handle, C.byref(ds.view), d_rays.data_ptr(), n,
                                        mcpt.ISECT_REFERENCE, d_hits.data_ptr()))
    mine = d_hits.cpu().numpy()
    assert np.array_equal(mine[:, 3], ref_hits[:, 3]), "did_hit"
    assert np.array_equal(mine[:, 2], ref_hits[:, 2]), "primitive index"
    assert np.array_equal(mine[:, 1], ref_hits[:, 1]), "primitive type"
    t_ulp = ulp_diff(mine[:, 0].view(np.float32), ref_hits[:, 0].view(np.float32))
    assert t_ulp.max() <= 2, t_ulp.max()
    assert mine[:, 3].mean() > 0.3  # the ray set does hit geometry


@pytest.mark.parametrize("kind,variant", CASES)
def test_any_hit_matches_reference(ctx, kind, variant):
    s = scene(kind, variant)
    tris = mcpt.host_triangles(s)
    r, ds, bvh = build_pair(ctx, tris, inject=True)
    ref = upload_ref(s)
    rays = random_rays(300000, -1.5, 1.5, seed=11) if kind == 2 else random_rays(300000, (-1.9, 0.1, -3.9), (1.9, 3.9, -0.1), seed=11)
    n = rays.shape[1]
    tmax = np.random.default_rng(3).uniform(0.01, 6.0, n).astype(np.float32)
    ref_occ = np.zeros(n, np.int32)
    assert ref.mcref_trace(rays.ctypes.data, n, 2, tmax.ctypes.data, None, ref_occ.ctypes.data) == 0
    occ = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_rays, d_tmax = dev(rays), dev(tmax)  # keep both alive across the call (torch reuses freed blocks)
    mcpt.check(ctx.lib.mc_trace_any(ctx.handle, bvh.handle, C.byref(ds.view), d_rays.data_ptr(), d_tmax.data_ptr(),
                                    n, mcpt.ISECT_REFERENCE, occ.data_ptr()))
    assert np.array_equal(occ.cpu().numpy(), ref_occ)
    assert 0.05 < ref_occ.mean() < 0.95


def render_mine(ctx, s, W, H, spp, depth, rng, inject=True, persistent=True, env=False):
    tris = mcpt.host_triangles(s)
    r = ref_sort(tris)
    e = mcpt.host_env(s) if env else None
    ds = mcpt.DeviceScene(tris, env_rgba=e, env_intensity=s.env_intensity)
    bvh = mcpt.Bvh(ctx, ds.view, permutation=dev(r["perm"]) if inject else None)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = W / float(H)
    mcpt.camera_initialize(cam)
    p = mcpt.render_params(cam, W, H, spp, depth, persistent=persistent, rng=rng, seed=1234)
    acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    st = mcpt.RenderStats()
    mcpt.check(ctx.lib.mc_rng_reset(ctx.handle, W, H, 1234))
    mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(), C.byref(st)))
    return acc.cpu().numpy().reshape(H, W, 3), st


def render_ref(s, W, H, spp, depth, mode, philox, unmodified=0, env=False):
    ref = mcref.load(philox)
    tris = mcpt.host_triangles(s)
    e = mcpt.host_env(s) if env else None
    assert ref.mcref_scene_upload(C.addressof(tris), len(tris), None, 0, e.ctypes.data if e is not None else None,
                                  s.env_width if e is not None else 0, s.env_height if e is not None else 0,
                                  s.env_intensity, 0.0) == 0
    acc = np.zeros(W * H * 3, np.float32)
    stats = np.zeros(3, np.float64)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    assert ref.mcref_render(C.addressof(cam), W, H, spp, depth, mode, 1234, 0, unmodified, acc.ctypes.data,
                            stats.ctypes.data) == 0
    return acc.reshape(H, W, 3), stats


def pixel_agreement(a, b, rel=1e-4):
    den = np.maximum(np.abs(b), 1e-6)
    ok = (np.abs(a - b) <= rel * den) | (np.abs(a - b) <= 1e-6)
    return ok.all(axis=2).mean()


@pytest.mark.parametrize("kind,variant,W,H,spp", [(mcpt.SCENE_CORNELL_BOXES, 0, 512, 512, 4),
                                                  (mcpt.SCENE_DISPLACED_ICOSPHERES, 5, 320, 180, 2)])
def test_image_parity_philox(ctx, kind, variant, W, H, spp):
    s = scene(kind, variant)
    env = kind == mcpt.SCENE_DISPLACED_ICOSPHERES
    mine, st = render_mine(ctx, s, W, H, spp, 8, mcpt.RNG_PHILOX, env=env)
    ref, rs = render_ref(s, W, H, spp, 8, 2, philox=True, env=env)
    frac = pixel_agreement(mine, ref)
    print("philox pixel agreement", frac, "exact", np.mean(np.all(mine == ref, axis=2)),
          "rays", st.extend_rays, st.shadow_rays, "ref rays", rs[0], rs[1])
    assert frac >= 0.999
    assert abs(st.extend_rays - rs[0]) <= 0.001 * rs[0]


def test_image_parity_xorwow_unmodified(ctx):
    """Against renderWithWavefront itself, curand XORWOW as in the reference."""
    s = scene(mcpt.SCENE_CORNELL_BOXES, 0)
    mine, st = render_mine(ctx, s, 512, 512, 2, 8, mcpt.RNG_XORWOW)
    ref, _ = render_ref(s, 512, 512, 2, 8, 2, philox=False, unmodified=1)
    frac = pixel_agreement(mine, ref)
    print("xorwow pixel agreement", frac)
    assert frac >= 0.999
