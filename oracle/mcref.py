"""ctypes binding of the oracle harness around the unmodified reference
(oracle/_ref/libmcref.so and libmcref_philox.so). Test infrastructure only:
imported by tests/, by tests/golden/make_golden.py and by bench.py's
reference arm. Built by oracle/Makefile (needs the reference sources); the
built .so files travel with the repository snapshot, the sources do not.
The harness also carries the library's seeded scene generator
(mcref_generate_scene), so the reference arm needs nothing else.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
P = C.c_void_p
I32 = C.c_int32

_SIGS = {
    "mcref_is_philox": (I32, []),
    "mcref_camera_initialize": (I32, [P]),
    "mcref_finalize_and_sort": (I32, [P, I32, P, I32, P, P, P, P, P, P, P, P, P, P]),
    "mcref_build_bvh": (I32, [P, P, P, P, I32, P, P]),
    "mcref_scene_upload": (I32, [P, I32, P, I32, P, I32, I32, C.c_float, C.c_float]),
    "mcref_scene_release": (I32, []),
    "mcref_trace": (I32, [P, I32, I32, P, P, P]),
    "mcref_render": (I32, [P, I32, I32, I32, I32, I32, C.c_ulonglong, I32, I32, P, P]),
    "mcref_resolve": (I32, [P, I32, I32, I32, I32, C.c_float, I32, P, P, P]),
    "mcref_load_object": (I32, [C.c_char_p, P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, P, I32, P]),
    "mcref_load_pfm": (I32, [C.c_char_p, P, P, P]),
    "mcref_generate_scene": (I32, [I32, I32, C.c_ulonglong, I32, P]),
    "mcref_free_scene": (I32, [P]),
    "mcref_grid_sample": (I32, [P, P, I32, P]),
    "mcref_cloud_scene": (I32, [P, P, C.c_float, C.c_uint64, I32, P, I32, P, P, I32, P]),
}
_libs = {}

# mc_scene_host (include/mc_abi.h) with the camera as its 172 raw bytes: the
# reference arm of the benchmark reads the seeded scenes through the harness
# without the library's Python binding.
SCENE_DISPLACED_ICOSPHERES = 2


class SceneHost(C.Structure):
    _fields_ = [("triangles", P), ("triangle_count", I32), ("spheres", P), ("sphere_count", I32),
                ("camera", C.c_float * 43), ("width", I32), ("height", I32), ("spp", I32), ("max_depth", I32),
                ("has_medium", I32), ("env_rgba", P), ("env_width", I32), ("env_height", I32),
                ("env_intensity", C.c_float)]


def path(philox=False):
    return os.path.join(HERE, "_ref", "libmcref_philox.so" if philox else "libmcref.so")


def available(philox=False):
    return os.path.exists(path(philox))


def load(philox=False):
    if philox in _libs:
        return _libs[philox]
    p = path(philox)
    if not os.path.exists(p):
        raise FileNotFoundError("oracle harness not built: %s (make -C oracle)" % p)
    lib = C.CDLL(p)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _libs[philox] = lib
    return lib


def addr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    return C.addressof(x)
