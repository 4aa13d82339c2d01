"""OBJ/MTL loading (mc_obj_load) and the PPM reader (mc_ppm_read) against the
reference's own loadObject (PT:2644-2859, with loadMtlFile PT:2614-2680),
run from oracle/_ref on the host.

Bar: bit-exact triangles (vertices, uvs, normals and every material field),
on files written here that exercise what the loader handles: v/vt/vn,
polygons (fan triangulation), negative and partial indices ("7//5", "7/3"),
out-of-range indices and zero-area faces (skipped), missing vn (area-weighted
vertex normals), zero-length vn, CRLF line ends, comments, materials with Kd,
Ke (emissive) and map_Kd (its image missing), unknown usemtl names, a missing
material library, and non-trivial scale, rotation and translation.
"""
import ctypes as C
import os

import numpy as np
import pytest

import mcpt
import mcref


def _sphere(subdiv, rng):
    """An octahedron subdivided `subdiv` times, projected to a bumpy sphere:
    vertex positions, uvs and per-vertex normals, triangle index list."""
    v = [np.array(p, float) for p in [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]]
    f = [(0, 2, 4), (2, 1, 4), (1, 3, 4), (3, 0, 4), (2, 0, 5), (1, 2, 5), (3, 1, 5), (0, 3, 5)]
    for _ in range(subdiv):
        cache, nf = {}, []
        for a, b, c in f:
            def mid(i, j):
                k = (min(i, j), max(i, j))
                if k not in cache:
                    cache[k] = len(v)
                    v.append((v[i] + v[j]) / 2)
                return cache[k]
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca)]
        f = nf
    P = np.array([p / np.linalg.norm(p) * (1 + 0.1 * rng.random()) for p in v])
    P = P * np.array([2.0, 1.0, 0.7]) + np.array([3.0, -1.0, 0.5])
    UV = rng.random((len(P), 2))
    N = P / np.linalg.norm(P, axis=1, keepdims=True)
    return P, UV, N, f


def _write(path, text, crlf=False):
    with open(path, "wb") as fh:
        fh.write(text.replace("\n", "\r\n" if crlf else "\n").encode())


def _reference(path, fallback, t, scale, rot):
    cap = 1 << 16
    out = (mcpt.Triangle * cap)()
    n = C.c_int32()
    rc = mcref.load(False).mcref_load_object(os.fsencode(path), C.byref(fallback), t[0], t[1], t[2], scale, rot,
                                             C.addressof(out), cap, C.byref(n))
    return rc, out, n.value


def _fields(tris, n):
    """Every value-carrying field of the first n triangles (padding excluded)."""
    rows = []
    for i in range(n):
        t = tris[i]
        m = t.mat
        rows.append(bytes(t)[:96] + bytes(C.c_int32(m.type)) + bytes(C.c_int32(m.albedo.type)) + bytes(m.albedo.color_a)
                    + bytes(m.albedo.color_b) + bytes(C.c_float(m.albedo.scale)) + bytes(C.c_uint64(m.albedo.image))
                    + bytes(m.emitted) + bytes(C.c_float(m.fuzz)) + bytes(C.c_float(m.refraction_index))
                    + bytes(C.c_float(m.density)) + bytes(C.c_float(m.phase_g))
                    + bytes(C.c_uint64(m.density_grid or 0)) + bytes(C.c_float(m.grid_max_density)))
    return rows


def _compare(path, t=(0.5, -0.25, 2.0), scale=1.7, rot=0.6, expect=None):
    fallback = mcpt.Material()
    fallback.type = mcpt.MAT_CONDUCTOR
    fallback.albedo.type = mcpt.TEX_SOLID
    fallback.albedo.color_a = mcpt.Vec3(0.3, 0.5, 0.7)
    fallback.albedo.scale = 1.0
    fallback.fuzz = 0.2
    rc, ref, rn = _reference(path, fallback, t, scale, rot)
    scene, info = mcpt.obj_load(path, fallback, t, scale, rot)
    try:
        assert rc == 0
        assert scene.triangle_count == rn == info.triangles_added
        mine = mcpt.host_triangles(scene)
        assert _fields(mine, rn) == _fields(ref, rn)
        if expect:
            for k, v in expect.items():
                assert getattr(info, k) == v, k
    finally:
        mcpt.obj_info_free(info)
        mcpt.free_scene(scene)
    return rn


def test_obj_with_normals_uvs_polygons_and_bad_faces(tmp_path):
    rng = np.random.default_rng(1)
    P, UV, N, F = _sphere(3, rng)
    lines = ["# a bumpy sphere", "o sphere", ""]
    lines += ["v %.7f %.7f %.7f" % tuple(p) for p in P]
    lines += ["vt %.6f %.6f" % tuple(u) for u in UV]
    lines += ["vn %.6f %.6f %.6f" % tuple(n) for n in N]
    lines.append("vn 0 0 0")  # zero length: the averaged / missing normal path
    nv = len(P)
    for k, (a, b, c) in enumerate(F):
        if k % 5 == 0:
            lines.append("f %d/%d/%d %d/%d/%d %d/%d/%d" % (a + 1, a + 1, a + 1, b + 1, b + 1, b + 1, c + 1, c + 1, c + 1))
        elif k % 5 == 1:
            lines.append("f %d//%d %d//%d %d//%d" % (a - nv, a - nv, b - nv, b - nv, c - nv, c - nv))  # negative
        elif k % 5 == 2:
            lines.append("f %d/%d %d/%d %d/%d" % (a + 1, a + 1, b + 1, b + 1, c + 1, c + 1))
        elif k % 5 == 3:
            lines.append("f %d %d %d" % (a + 1, b + 1, c + 1))
        else:
            lines.append("f %d//%d %d//%d %d//%d" % (a + 1, nv + 1, b + 1, nv + 1, c + 1, nv + 1))  # zero vn
    lines.append("f 1 2 3 4 5 6")            # a hexagon: 4 fan triangles
    lines.append("f 1 1 1")                  # zero area: skipped
    lines.append("f 1 2 %d" % (nv + 50))     # index out of range: skipped
    lines.append("f 1 2 0")                  # index 0 is invalid: skipped
    p = str(tmp_path / "sphere.obj")
    _write(p, "\n".join(lines) + "\n", crlf=True)
    n = _compare(p, expect={"faces_skipped": 3})
    assert n == len(F) + 4


def test_obj_without_normals_uses_area_weighted_vertex_normals(tmp_path):
    rng = np.random.default_rng(2)
    P, UV, N, F = _sphere(2, rng)
    lines = ["v %.7f %.7f %.7f" % tuple(p) for p in P] + ["f %d %d %d" % (a + 1, b + 1, c + 1) for a, b, c in F]
    p = str(tmp_path / "plain.obj")
    _write(p, "\n".join(lines))
    _compare(p, t=(0, 0, 0), scale=1.0, rot=0.0)
    _compare(p, t=(-4, 2, 1), scale=0.25, rot=-2.5)


def test_obj_materials_from_mtl(tmp_path):
    _write(str(tmp_path / "a.mtl"), "\n".join([
        "# library", "newmtl red", "Kd 0.8 0.1 0.1", "Ka 1 1 1",
        "newmtl lamp", "Kd 0.5 0.5 0.5", "Ke 4 3.5 2",
        "newmtl wall", "Kd 0.2 0.6 0.3", "map_Kd textures\\\\wall.png",
        "newmtl grey"]) + "\n")
    rng = np.random.default_rng(3)
    P, UV, N, F = _sphere(2, rng)
    lines = ["mtllib a.mtl missing.mtl"] + ["v %.7f %.7f %.7f" % tuple(p) for p in P]
    names = ["red", "lamp", "wall", "grey", "nosuch", None]
    for k, (a, b, c) in enumerate(F):
        if k % 17 == 0:
            nm = names[(k // 17) % len(names)]
            if nm:
                lines.append("usemtl " + nm)
        lines.append("f %d %d %d" % (a + 1, b + 1, c + 1))
    p = str(tmp_path / "mat.obj")
    _write(p, "\n".join(lines) + "\n")
    _compare(p, expect={"materials": 4, "textures_missing": 1, "textures_loaded": 0, "unknown_materials": 1})


def test_obj_with_one_material_uses_it_for_unknown_names(tmp_path):
    _write(str(tmp_path / "one.mtl"), "newmtl only\nKd 0.1 0.2 0.9\n")
    _write(str(tmp_path / "one.obj"), "mtllib one.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nusemtl other\nf 1 2 3\nf 1 3 4\n")
    _compare(str(tmp_path / "one.obj"))


def test_obj_errors(tmp_path):
    fb = mcpt.Material()
    lib = mcpt.load()
    sc = mcpt.SceneHost()
    info = mcpt.ObjInfo()
    assert mcpt.STATUS_NAMES[lib.mc_obj_load(os.fsencode(str(tmp_path / "none.obj")), C.byref(fb), mcpt.Vec3(0, 0, 0),
                                             1.0, 0.0, 0, C.byref(sc), C.byref(info))] == "MC_ERR_NOT_FOUND"
    _write(str(tmp_path / "empty.obj"), "# nothing\nv 0 0 0\n")
    assert mcpt.STATUS_NAMES[lib.mc_obj_load(os.fsencode(str(tmp_path / "empty.obj")), C.byref(fb), mcpt.Vec3(0, 0, 0),
                                             1.0, 0.0, 0, C.byref(sc), C.byref(info))] == "MC_ERR_INVALID"
    _write(str(tmp_path / "flat.obj"), "v 0 0 0\nv 1 0 0\nv 2 0 0\nf 1 2 3\n")  # every face has zero area
    assert mcpt.STATUS_NAMES[lib.mc_obj_load(os.fsencode(str(tmp_path / "flat.obj")), C.byref(fb), mcpt.Vec3(0, 0, 0),
                                             1.0, 0.0, 0, C.byref(sc), C.byref(info))] == "MC_ERR_INVALID"
    assert sc.triangle_count == 0
    mcpt.free_scene(sc)


def test_obj_appends_to_a_generated_scene(tmp_path):
    _write(str(tmp_path / "t.obj"), "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
    n0 = s.triangle_count
    before = bytes(mcpt.host_triangles(s))
    s, info = mcpt.obj_load(str(tmp_path / "t.obj"), mcpt.Material(), scene=s)
    assert s.triangle_count == n0 + 1 and info.triangles_added == 1
    assert bytes(mcpt.host_triangles(s))[:len(before)] == before
    mcpt.obj_info_free(info)
    mcpt.free_scene(s)


def test_ppm_reader(tmp_path):
    rng = np.random.default_rng(4)
    px = rng.integers(0, 256, (7, 11, 3), dtype=np.uint8)
    p = str(tmp_path / "a.ppm")
    with open(p, "wb") as fh:
        fh.write(b"P6\n# a comment\n11 7\n# another\n255\n" + px.tobytes())
    w, h = C.c_int32(), C.c_int32()
    lib = mcpt.load()
    mcpt.check(lib.mc_ppm_read(os.fsencode(p), C.byref(w), C.byref(h), None))
    assert (w.value, h.value) == (11, 7)
    out = np.zeros(11 * 7 * 4, np.uint8)
    mcpt.check(lib.mc_ppm_read(os.fsencode(p), C.byref(w), C.byref(h), out.ctypes.data))
    got = out.reshape(7, 11, 4)
    assert np.array_equal(got[..., :3], px) and (got[..., 3] == 255).all()
    for bad in [b"P5\n11 7\n255\n", b"P6\n11 7\n65535\n", b"P6\n11 7\n255\n" + px.tobytes()[:-1]]:
        with open(p, "wb") as fh:
            fh.write(bad + (px.tobytes() if bad.startswith(b"P5") else b""))
        assert lib.mc_ppm_read(os.fsencode(p), C.byref(w), C.byref(h), out.ctypes.data) == 1
