"""Host file readers (no GPU): mc_pfm_read against the reference's own
loadPfmAsRgba32f (src/path_tracer.cu:335-368, run from oracle/_ref) on valid
files and on the edge cases its rules decide; the dense grid files of
--volume; and the command-line driver's handling of --env, --volume, --pbrt
before any device work."""
import ctypes as C
import os
import struct
import subprocess

import numpy as np
import pytest

import mcpt
import mcref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "monocuda-pt_b200", "monocuda")


def _pfm(header, w, h, pixels=None, extra=b""):
    if pixels is None:
        pixels = np.random.default_rng(w * 31 + h).normal(0, 3, (h, w, 3)).astype("<f4")
    return header + np.ascontiguousarray(pixels, "<f4").tobytes() + extra


CASES = {
    "standard": _pfm(b"PF\n5 3\n-1.0\n", 5, 3),
    "one line": _pfm(b"PF 4 2 -1\n", 4, 2),
    "spaces": _pfm(b"PF\n\n 4   2\n  -1.000\n", 4, 2),
    "scale zero": _pfm(b"PF\n3 3\n0\n", 3, 3),
    "trailing data": _pfm(b"PF\n2 2\n-1.0\n", 2, 2, extra=b"tail"),
    "one pixel": _pfm(b"PF\n1 1\n-1.0\n", 1, 1),
    "big endian": _pfm(b"PF\n3 2\n1.0\n", 3, 2),
    "greyscale": b"Pf\n3 2\n-1.0\n" + bytes(24),
    "magic too long": _pfm(b"PFX\n3 2\n-1.0\n", 3, 2),
    "zero width": b"PF\n0 2\n-1.0\n",
    "truncated": _pfm(b"PF\n4 4\n-1.0\n", 4, 4)[:-5],
    "no separator": b"PF\n4 4\n-1.0",
    "text": b"hello world\n",
}


def _reference(path):
    lib = mcref.load(False)
    w, h = C.c_int32(), C.c_int32()
    if lib.mcref_load_pfm(path.encode(), C.byref(w), C.byref(h), None) != 0:
        return None
    out = np.zeros((h.value, w.value, 4), np.float32)
    assert lib.mcref_load_pfm(path.encode(), C.byref(w), C.byref(h), out.ctypes.data) == 0
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_pfm_reader_matches_reference(tmp_path, name):
    path = os.path.join(tmp_path, "e.pfm")
    with open(path, "wb") as f:
        f.write(CASES[name])
    ref = _reference(path)
    try:
        mine = mcpt.pfm_read(path)
    except mcpt.McError:
        mine = None
    assert (mine is None) == (ref is None), name
    if ref is not None:
        assert mine.shape == ref.shape and np.array_equal(mine.view(np.uint32), ref.view(np.uint32)), name


def test_pfm_rows_and_alpha(tmp_path):
    path = os.path.join(tmp_path, "g.pfm")
    px = np.arange(2 * 3 * 3, dtype=np.float32).reshape(2, 3, 3)  # file order: bottom row first
    with open(path, "wb") as f:
        f.write(b"PF\n3 2\n-1.0\n" + px.astype("<f4").tobytes())
    img = mcpt.pfm_read(path)
    assert np.array_equal(img[..., :3], px[::-1]) and np.all(img[..., 3] == 1.0)


def test_pfm_missing_file():
    with pytest.raises(mcpt.McError):
        mcpt.pfm_read("/nonexistent/e.pfm")


def test_volume_file_round_trip(tmp_path):
    rng = np.random.default_rng(4)
    d = rng.random((5, 7, 9)).astype(np.float32)
    path = os.path.join(tmp_path, "g.mcvol")
    mcpt.volume_file_write(path, d, (0.1, -2.0, 3.5), 0.07)
    got, org, voxel = mcpt.volume_file_read(path)
    assert np.array_equal(got, d)
    assert org == tuple(np.float32(x) for x in (0.1, -2.0, 3.5)) and voxel == np.float32(0.07)
    with open(path, "rb") as f:
        assert f.readline().split()[:4] == [b"MCVOL", b"9", b"7", b"5"]


@pytest.mark.parametrize("content", [b"MCVOX 2 2 2 0.1 0 0 0\n", b"MCVOL 0 2 2 0.1 0 0 0\n", b"MCVOL 2 2 2 -1 0 0 0\n",
                                     b"MCVOL 2 2 2 0.1 0 0 0\n" + bytes(8), b"MCVOL 2 2 2 0.1 0 0 0 " + bytes(32)])
def test_volume_file_rejects_bad_files(tmp_path, content):
    path = os.path.join(tmp_path, "bad.mcvol")
    with open(path, "wb") as f:
        f.write(content)
    with pytest.raises(mcpt.McError):
        mcpt.volume_file_read(path)


def _run(*args):
    return subprocess.run([CLI] + list(args), capture_output=True, text=True, timeout=120)


@pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built")
def test_cli_refuses_what_it_cannot_read(tmp_path):
    r = _run("--pbrt", "scene.pbrt")
    assert r.returncode == 2 and "pbrt scene import" in r.stderr
    r = _run("--max-triangles", "100")
    assert r.returncode == 2
    r = _run("--wavefront", "--env", os.path.join(tmp_path, "sky.hdr"))
    assert r.returncode == 1 and "only PFM" in r.stderr
    r = _run("--wavefront", "--env", os.path.join(tmp_path, "missing.pfm"))
    assert r.returncode == 1 and "environment map" in r.stderr
    bad = os.path.join(tmp_path, "bad.pfm")
    with open(bad, "wb") as f:
        f.write(CASES["big endian"])
    r = _run("--wavefront", "--env", bad)
    assert r.returncode == 1 and "big-endian" in r.stderr
    r = _run("--wavefront", "--volume", os.path.join(tmp_path, "missing.mcvol"))
    assert r.returncode == 1 and "volume" in r.stderr
    r = _run("--wavefront", "--scene", "cloud")
    assert r.returncode == 1 and "needs a density grid" in r.stderr
    r = _run("--help")
    assert r.returncode == 0 and "--env" in r.stdout and "--phase-g" in r.stdout and "--volume" in r.stdout
