"""Parity on the benchmarked workload itself: the 3,932,176-triangle displaced
icospheres scene at 1920x1080, traversed through the build the benchmark uses
(clustered binary tree collapsed to the 4-wide layout), against the UNMODIFIED
reference (oracle/_ref) on the same GPU.

Bars: closest-hit primitive ids and types bit-exact, t within 2 ulp, any-hit
answers equal (reference extendKernelPersistent PT:3416-3468 and
traverseAnyHit PT:1152-1207 on the same rays); the image of a 2-spp render
with the library's automatic samples per wave within 1e-4 relative on EVERY
pixel of the reference's renderWithWavefront (PT:3757-3840) under the shared
counter-based RNG, and the same ray counts.
"""
import ctypes as C

import numpy as np
import pytest

import mcpt
import mcref
from helpers import primary_rays, random_rays, ulp_diff

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ICO = mcpt.SCENE_DISPLACED_ICOSPHERES


@pytest.fixture(scope="module")
def bench_setup():
    ctx = mcpt.Context(0)
    s = mcpt.generate_scene(ICO, variant=8, seed=2)
    tris = mcpt.host_triangles(s)
    n = len(tris)
    assert n == 3932176
    ref = mcref.load()
    perm = np.zeros(n, np.int32)
    scratch = {k: np.zeros(n, np.uint32) for k in ("codes", "sorted")}
    ids, types = np.zeros(n, np.int32), np.zeros(n, np.int32)
    sb, bb = np.zeros(n * 8, np.float32), np.zeros(8, np.float32)
    tb, lights = np.zeros(n * 8, np.float32), np.zeros(n * 16, np.float32)
    nl = C.c_int32()
    assert ref.mcref_finalize_and_sort(C.addressof(tris), n, None, 0, scratch["codes"].ctypes.data,
                                       scratch["sorted"].ctypes.data, ids.ctypes.data, types.ctypes.data,
                                       perm.ctypes.data, sb.ctypes.data, bb.ctypes.data, tb.ctypes.data,
                                       lights.ctypes.data, C.byref(nl)) == 0
    del scratch, ids, types, sb, tb, lights
    env = mcpt.host_env(s)
    ds = mcpt.DeviceScene(tris, env_rgba=env, env_intensity=s.env_intensity)
    d_perm = torch.from_numpy(perm).cuda()
    bvh = mcpt.Bvh(ctx, ds.view, permutation=d_perm, layout=mcpt.LAYOUT_WIDE4, builder=mcpt.BUILDER_CLUSTERED)
    del d_perm
    yield ctx, s, tris, env, ds, bvh
    bvh.close()
    ctx.close()


def upload_reference(s, tris, env, philox):
    ref = mcref.load(philox)
    assert ref.mcref_scene_upload(C.addressof(tris), len(tris), None, 0, env.ctypes.data, s.env_width, s.env_height,
                                  s.env_intensity, 0.0) == 0
    return ref


def bench_rays(s):
    """Every primary ray of the 1920x1080 image plus one million random rays
    (origins around and inside the three spheres, directions on the sphere)."""
    prim = primary_rays(s.camera, s.width, s.height, stride=1)
    rnd = random_rays(1000000, -3.0, 3.0, seed=31)
    return np.ascontiguousarray(np.concatenate([prim, rnd], axis=1))


def test_bench_scene_closest_hits_match_reference(bench_setup):
    ctx, s, tris, env, ds, bvh = bench_setup
    assert bvh.info().layout == mcpt.LAYOUT_WIDE4
    ref = upload_reference(s, tris, env, philox=False)
    rays = bench_rays(s)
    n = rays.shape[1]
    assert n >= 3_000_000
    ref_hits = np.zeros((n, 4), np.int32)
    assert ref.mcref_trace(rays.ctypes.data, n, 0, None, ref_hits.ctypes.data, None) == 0
    d_rays = torch.from_numpy(rays).cuda()
    d_hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    mcpt.check(ctx.lib.mc_trace_closest(ctx.handle, bvh.handle, C.byref(ds.view), d_rays.data_ptr(), n,
                                        mcpt.ISECT_REFERENCE, d_hits.data_ptr()))
    mine = d_hits.cpu().numpy()
    assert np.array_equal(mine[:, 3], ref_hits[:, 3]), "did_hit differs on %d rays" % int((mine[:, 3] != ref_hits[:, 3]).sum())
    bad = mine[:, 2] != ref_hits[:, 2]
    assert not bad.any(), "primitive index differs on %d of %d rays" % (int(bad.sum()), n)
    assert np.array_equal(mine[:, 1], ref_hits[:, 1]), "primitive type"
    t_ulp = ulp_diff(mine[:, 0].view(np.float32), ref_hits[:, 0].view(np.float32))
    print("bench scene: %d rays, hit fraction %.3f, max t difference %d ulp" % (n, ref_hits[:, 3].mean(), t_ulp.max()))
    assert t_ulp.max() <= 2
    assert ref_hits[:, 3].mean() > 0.3


def test_bench_scene_any_hit_matches_reference(bench_setup):
    ctx, s, tris, env, ds, bvh = bench_setup
    ref = upload_reference(s, tris, env, philox=False)
    rays = bench_rays(s)
    n = rays.shape[1]
    tmax = np.random.default_rng(32).uniform(0.01, 8.0, n).astype(np.float32)
    ref_occ = np.zeros(n, np.int32)
    assert ref.mcref_trace(rays.ctypes.data, n, 2, tmax.ctypes.data, None, ref_occ.ctypes.data) == 0
    d_rays, d_tmax = torch.from_numpy(rays).cuda(), torch.from_numpy(tmax).cuda()
    occ = torch.zeros(n, dtype=torch.int32, device="cuda")
    mcpt.check(ctx.lib.mc_trace_any(ctx.handle, bvh.handle, C.byref(ds.view), d_rays.data_ptr(), d_tmax.data_ptr(),
                                    n, mcpt.ISECT_REFERENCE, occ.data_ptr()))
    mine = occ.cpu().numpy()
    assert np.array_equal(mine, ref_occ), "any-hit answer differs on %d rays" % int((mine != ref_occ).sum())
    assert 0.05 < ref_occ.mean() < 0.95


def test_bench_scene_image_matches_reference(bench_setup):
    """1920x1080, 2 spp, depth 8, the sky and the medium box: the library's
    automatic samples per wave (pixel-major) against the reference's
    renderWithWavefront with the same Philox stream per (pixel, sample)."""
    ctx, s, tris, env, ds, bvh = bench_setup
    W, H, spp = s.width, s.height, 2
    assert (W, H) == (1920, 1080)
    p = mcpt.render_params(s.camera, W, H, spp, 8, persistent=True, rng=mcpt.RNG_PHILOX, seed=1234)
    acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    st = mcpt.RenderStats()
    mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                           C.byref(st)))
    mine = acc.cpu().numpy().reshape(H, W, 3)
    ref = upload_reference(s, tris, env, philox=True)
    racc = np.zeros(W * H * 3, np.float32)
    stats = np.zeros(3, np.float64)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    assert ref.mcref_render(C.addressof(cam), W, H, spp, 8, 2, 1234, 0, 0, racc.ctypes.data, stats.ctypes.data) == 0
    racc = racc.reshape(H, W, 3)
    diff = np.abs(mine - racc)
    ok = (diff <= 1e-4 * np.maximum(np.abs(racc), 1e-6)) | (diff <= 1e-6)
    bad = int((~ok.all(axis=2)).sum())
    print("bench scene image: %d of %d pixels outside 1e-4, identical %.6f, rays %d+%d (reference %d+%d)"
          % (bad, W * H, np.mean(np.all(mine == racc, axis=2)), st.extend_rays, st.shadow_rays, stats[0], stats[1]))
    assert bad == 0
    assert abs(st.extend_rays - stats[0]) <= 1e-3 * stats[0] and abs(st.shadow_rays - stats[1]) <= 1e-3 * stats[1]
