"""An OBJ mesh with an image texture (mc_obj_load with textures, mc_image_texture_create)
rendered in the Cornell boxes scene: the image equals the reference's
renderWithWavefront on the same triangles (same texture objects), per pixel
within 1e-4 relative, as the other image-parity tests."""
import os

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


def _write_textured_mesh(d):
    rng = np.random.default_rng(8)
    img = rng.integers(0, 256, (32, 64, 3), dtype=np.uint8)
    with open(os.path.join(d, "checker.ppm"), "wb") as fh:
        fh.write(b"P6\n64 32\n255\n" + img.tobytes())
    with open(os.path.join(d, "m.mtl"), "w") as fh:
        fh.write("newmtl tex\nKd 0.9 0.9 0.9\nmap_Kd checker.png\nnewmtl glow\nKe 2 2 1.5\n")
    # a UV sphere with seams: latitude/longitude grid
    nu, nv = 24, 12
    lines = ["mtllib m.mtl"]
    for j in range(nv + 1):
        th = np.pi * j / nv
        for i in range(nu + 1):
            ph = 2 * np.pi * i / nu
            lines.append("v %.6f %.6f %.6f" % (np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)))
            lines.append("vt %.6f %.6f" % (i / nu * 2.0, j / nv))
    lines.append("usemtl tex")
    for j in range(nv):
        for i in range(nu):
            a = j * (nu + 1) + i + 1
            b, c, e = a + 1, a + nu + 1, a + nu + 2
            if j == nv - 1 and i % 6 == 0:
                lines.append("usemtl glow")
            lines.append("f %d/%d %d/%d %d/%d %d/%d" % (a, a, b, b, e, e, c, c))
            if j == nv - 1 and i % 6 == 0:
                lines.append("usemtl tex")
    with open(os.path.join(d, "ball.obj"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return os.path.join(d, "ball.obj")


@pytest.mark.parametrize("layout", [mcpt.LAYOUT_BINARY, mcpt.LAYOUT_WIDE4])
def test_textured_obj_image_parity(ctx, tmp_path, layout):
    path = _write_textured_mesh(str(tmp_path))
    fallback = mcpt.Material()
    images = {}
    for textures in (True, False):
        s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
        s, info = mcpt.obj_load(path, fallback, translation=(0.1, 0.0, -1.3), scale=0.9, rotation_y=0.4,
                                load_textures=textures, scene=s)
        assert info.textures_loaded == (1 if textures else 0)
        assert info.textures_missing == (0 if textures else 1)
        mine, st = render_mine(ctx, s, 192, 192, 4, 8, mcpt.RNG_PHILOX, layout=layout)
        ref, rs = render_ref(s, 192, 192, 4, 8, 2, philox=True)
        frac = pixel_agreement(mine, ref)
        print("textures %s layout %d: pixel agreement %.6f" % (textures, layout, frac))
        assert frac >= 0.999
        images[textures] = mine
        mcpt.obj_info_free(info)
        mcpt.free_scene(s)
    # the texture shows in the image
    assert np.abs(images[True] - images[False]).mean() > 1e-3
