"""ctypes binding of the C ABI in include/mc_abi.h (libmcpt.so, built in-tree).

The library is the product; this module only mirrors its structs and entry
points for Python callers (tests, bench.py, the render server driver). It
raises McError on any non-OK status and never falls back to anything else:
if libmcpt.so is missing or no GPU is present, the calls fail loudly.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmcpt.so")

MC_OK = 0
STATUS_NAMES = {0: "MC_OK", 1: "MC_ERR_INVALID", 2: "MC_ERR_CUDA", 3: "MC_ERR_OOM", 4: "MC_ERR_STACK_OVERFLOW",
                5: "MC_ERR_QUEUE_OVERFLOW", 6: "MC_ERR_TIMEOUT", 7: "MC_ERR_BUDGET", 8: "MC_ERR_CANCELLED",
                9: "MC_ERR_NOT_FOUND", 10: "MC_ERR_UNSUPPORTED"}
MAT_LAMBERTIAN, MAT_DIELECTRIC, MAT_CONDUCTOR, MAT_EMISSIVE, MAT_ISOTROPIC = 0, 1, 2, 3, 4
TEX_SOLID, TEX_CHECKER, TEX_IMAGE = 0, 1, 2
RNG_PHILOX, RNG_XORWOW = 0, 1
ISECT_REFERENCE, ISECT_WATERTIGHT = 0, 1
ENV_SAMPLE_CDF, ENV_SAMPLE_ALIAS = 0, 1
GUIDE_DIR_NORMAL, GUIDE_DIR_RAY = 0, 1
TRACE_PLAIN = 0x100
LAYOUT_BINARY, LAYOUT_WIDE4, LAYOUT_WIDE4Q = 0, 1, 2
BUILDER_CLUSTERED, BUILDER_LBVH = 0, 1
TONEMAP_NONE, TONEMAP_REINHARD, TONEMAP_ACES = 0, 1, 2
IMAGE_RGB8, IMAGE_RGB_F32, IMAGE_PFM, IMAGE_PNG = 0, 1, 2, 3
SCENE_CORNELL_BOXES, SCENE_DISPLACED_ICOSPHERES, SCENE_BATCH_MEMBER, SCENE_GUIDING_ROOM = 1, 2, 3, 4
SCENE_CORNELL_SPHERES = 5
MAX_DEPTH_STATS = 64
REQ_PENDING, REQ_ACTIVE, REQ_DONE, REQ_RELEASED, REQ_CANCELLED = 0, 1, 2, 3, 4
SORT_STATIC_MAX_PAIRS = 1 << 20
GUIDE_PARAM_COUNT = 20200
GUIDE_INPUTS, GUIDE_HIDDEN, GUIDE_OUTPUTS, GUIDE_LOBES = 144, 64, 40, 8


class McError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class Vec2(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float)]


class AABB(C.Structure):
    _fields_ = [("lo", Vec3), ("pad0", C.c_float), ("hi", Vec3), ("pad1", C.c_float)]


class Texture(C.Structure):
    _fields_ = [("type", C.c_int32), ("color_a", Vec3), ("color_b", Vec3), ("scale", C.c_float), ("image", C.c_uint64)]


class Material(C.Structure):
    _fields_ = [("type", C.c_int32), ("albedo", Texture), ("emitted", Vec3), ("fuzz", C.c_float),
                ("refraction_index", C.c_float), ("density", C.c_float), ("phase_g", C.c_float),
                ("density_grid", C.c_void_p), ("grid_max_density", C.c_float)]


class Triangle(C.Structure):
    _fields_ = [("v0", Vec3), ("v1", Vec3), ("v2", Vec3), ("uv0", Vec2), ("uv1", Vec2), ("uv2", Vec2),
                ("n0", Vec3), ("n1", Vec3), ("n2", Vec3), ("mat", Material), ("aabb", AABB)]


class TriangleHot(C.Structure):
    _fields_ = [("v0", Vec3), ("v1", Vec3), ("v2", Vec3)]


class TriangleCold(C.Structure):
    _fields_ = [("uv0", Vec2), ("uv1", Vec2), ("uv2", Vec2), ("n0", Vec3), ("n1", Vec3), ("n2", Vec3),
                ("mat", Material), ("aabb", AABB)]


class Sphere(C.Structure):
    _fields_ = [("center", Vec3), ("center1", Vec3), ("is_moving", C.c_uint8), ("radius", C.c_float),
                ("mat", Material), ("aabb", AABB)]


class Light(C.Structure):
    _fields_ = [("tri", TriangleHot), ("emitted", Vec3), ("area", C.c_float), ("normal", Vec3)]


class BvhNode(C.Structure):
    _fields_ = [("bounds", AABB), ("left", C.c_int32), ("right", C.c_int32), ("left_is_leaf", C.c_uint8),
                ("right_is_leaf", C.c_uint8), ("parent", C.c_int32), ("prim", C.c_int32), ("is_leaf", C.c_uint8),
                ("_tail", C.c_uint8 * 11)]  # the C struct is 16-byte aligned (it holds an AABB): 64 bytes


class PackedHit(C.Structure):
    _fields_ = [("t", C.c_float), ("type", C.c_int32), ("index", C.c_int32), ("did_hit", C.c_int32)]


class Camera(C.Structure):
    _fields_ = [("aspect_ratio", C.c_float), ("image_width", C.c_int32), ("image_height", C.c_int32),
                ("samples_per_pixel", C.c_int32), ("max_depth", C.c_int32), ("vfov", C.c_float),
                ("look_from", Vec3), ("look_at", Vec3), ("up", Vec3), ("center", Vec3), ("pixel00", Vec3),
                ("pixel_delta_u", Vec3), ("pixel_delta_v", Vec3), ("u", Vec3), ("v", Vec3), ("w", Vec3),
                ("background", Vec3), ("aperture", C.c_float), ("lens_radius", C.c_float),
                ("focus_distance", C.c_float), ("rr_cap", C.c_float)]


class VolumeGrid(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("voxel_size", C.c_float), ("inv_voxel_size", C.c_float),
                ("dims", C.c_int32 * 3), ("maximum_density", C.c_float), ("world_min", C.c_float * 3),
                ("world_max", C.c_float * 3), ("pad0", C.c_int32)]


MEDIUM_ANY, MEDIUM_GRID = 1, 2


class EnvMap(C.Structure):
    _fields_ = [("texture", C.c_uint64), ("enabled", C.c_int32), ("intensity", C.c_float), ("rotation", C.c_float),
                ("row_cdf", C.c_void_p), ("col_cdf", C.c_void_p), ("width", C.c_int32), ("height", C.c_int32),
                ("total_weight", C.c_float)]


class SceneView(C.Structure):
    _fields_ = [("spheres", C.c_void_p), ("sphere_count", C.c_int32), ("tri_hot", C.c_void_p), ("tri_cold", C.c_void_p),
                ("triangle_count", C.c_int32), ("lights", C.c_void_p), ("light_count", C.c_int32),
                ("has_medium", C.c_int32), ("env", EnvMap)]


class BvhBuildOpts(C.Structure):
    _fields_ = [("permutation", C.c_void_p), ("layout", C.c_int32), ("keep_reference_nodes", C.c_int32),
                ("builder", C.c_int32), ("phase_launches", C.c_int32)]


class BvhInfo(C.Structure):
    _fields_ = [("primitive_count", C.c_int32), ("internal_count", C.c_int32), ("depth", C.c_int32),
                ("layout", C.c_int32), ("node_bytes", C.c_int64), ("prim_bytes", C.c_int64), ("scene_bounds", AABB),
                ("wide_levels", C.c_int32)]


class RenderParams(C.Structure):
    _fields_ = [("camera", Camera), ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32),
                ("first_sample", C.c_int32), ("max_depth", C.c_int32), ("persistent", C.c_int32), ("rng", C.c_int32),
                ("seed", C.c_uint64), ("intersector", C.c_int32), ("disable_clamp", C.c_int32),
                ("queue_capacity", C.c_int32), ("refill_threshold", C.c_int32), ("use_graph", C.c_int32),
                ("instrument", C.c_int32), ("samples_per_wave", C.c_int32), ("env_sampling", C.c_int32),
                ("stack_entries", C.c_int32), ("trace_threads", C.c_int32)]


GUIDE_LOBES_ANCHORED = 1
GUIDE_LOBES_RAW = 2


class GuideConfig(C.Structure):
    _fields_ = [("bounds", AABB), ("learning_rate", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
                ("epsilon", C.c_float), ("seed", C.c_uint64), ("batch_capacity", C.c_int32),
                ("guide_fraction", C.c_float), ("train_steps", C.c_int32), ("train_vertices", C.c_int32),
                ("direction_input", C.c_int32), ("guided_depth", C.c_int32), ("weight_cap", C.c_float),
                ("fold_below", C.c_int32), ("anchor_lobes", C.c_int32), ("nee_records", C.c_int32)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("max_active", C.c_int32), ("samples_per_step", C.c_int32),
                ("wave_paths", C.c_int64), ("flags", C.c_int32), ("pad0", C.c_int32)]


SERVER_SCENE_WAVES = 1


class ServerRequest(C.Structure):
    _fields_ = [("scene_id", C.c_int64), ("params", RenderParams), ("guided", C.c_int32)]


class ServerResult(C.Structure):
    _fields_ = [("request_id", C.c_int64), ("state", C.c_int32), ("spp_done", C.c_int32), ("submit_s", C.c_double),
                ("admit_s", C.c_double), ("done_s", C.c_double), ("bytes", C.c_int64), ("d_accum", C.c_void_p)]


class ImageOptions(C.Structure):
    _fields_ = [("format", C.c_int32), ("tonemap", C.c_int32), ("exposure", C.c_float), ("device_output", C.c_int32)]


class ObjInfo(C.Structure):
    _fields_ = [("triangles_added", C.c_int32), ("faces_skipped", C.c_int32), ("materials", C.c_int32),
                ("textures_loaded", C.c_int32), ("textures_missing", C.c_int32), ("unknown_materials", C.c_int32),
                ("textures", C.POINTER(C.c_uint64))]


class ServerStats(C.Structure):
    _fields_ = [("budget_bytes", C.c_int64), ("used_bytes", C.c_int64), ("scene_bytes", C.c_int64),
                ("scenes", C.c_int32), ("pending", C.c_int32), ("active", C.c_int32), ("done", C.c_int32),
                ("steps", C.c_int64), ("waves", C.c_int64), ("rays", C.c_int64)]


class RenderStats(C.Structure):
    _fields_ = [("extend_rays", C.c_int64), ("shadow_rays", C.c_int64), ("paths", C.c_int64),
                ("extend_per_depth", C.c_int64 * MAX_DEPTH_STATS), ("shadow_per_depth", C.c_int64 * MAX_DEPTH_STATS),
                ("node_visits", C.c_int64), ("leaf_tests", C.c_int64), ("render_ms", C.c_float), ("trace_ms", C.c_float),
                ("trace_launches", C.c_int32), ("kernel_launches", C.c_int32), ("error_flags", C.c_int32),
                ("shade_ms", C.c_float), ("guide_infer_ms", C.c_float), ("guide_train_ms", C.c_float)]


class BatchItem(C.Structure):
    _fields_ = [("scene", SceneView), ("params", RenderParams), ("d_accum", C.c_void_p)]


class SceneDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("variant", C.c_int32), ("seed", C.c_uint64), ("triangle_target", C.c_int32)]


class SceneHost(C.Structure):
    _fields_ = [("triangles", C.POINTER(Triangle)), ("triangle_count", C.c_int32), ("spheres", C.POINTER(Sphere)),
                ("sphere_count", C.c_int32), ("camera", Camera), ("width", C.c_int32), ("height", C.c_int32),
                ("spp", C.c_int32), ("max_depth", C.c_int32), ("has_medium", C.c_int32),
                ("env_rgba", C.POINTER(C.c_float)), ("env_width", C.c_int32), ("env_height", C.c_int32),
                ("env_intensity", C.c_float)]


SIZES = {Vec3: 12, AABB: 32, Texture: 40, Material: 96, Triangle: 224, TriangleHot: 36, TriangleCold: 192,
         Sphere: 160, Light: 64, BvhNode: 64, PackedHit: 16, Camera: 172, EnvMap: 56, VolumeGrid: 64, GuideConfig: 96, RenderParams: 248,
         ServerConfig: 32, ServerRequest: 264, ServerResult: 56, ServerStats: 64}
for _t, _s in SIZES.items():
    assert C.sizeof(_t) == _s, (_t.__name__, C.sizeof(_t), _s)

P = C.c_void_p
I32 = C.c_int32
# name -> (restype, argtypes); every function declared in include/mc_abi.h
SIGNATURES = {
    "mc_version": (C.c_char_p, []),
    "mc_status_string": (C.c_char_p, [I32]),
    "mc_last_error": (C.c_char_p, []),
    "mc_context_create": (I32, [I32, C.POINTER(P)]),
    "mc_context_destroy": (I32, [P]),
    "mc_context_set_stream": (I32, [P, P]),
    "mc_context_synchronize": (I32, [P]),
    "mc_context_set_wait_timeout": (I32, [P, C.c_int64]),
    "mc_stream_wait_value": (I32, [P, P, C.c_uint32]),
    "mc_camera_initialize": (I32, [C.POINTER(Camera)]),
    "mc_scene_finalize_host": (I32, [P, I32, P, C.POINTER(I32)]),
    "mc_split_triangles_host": (I32, [P, I32, P, P]),
    "mc_scene_ingest": (I32, [P, P, I32, P, I32, P, P, P, C.POINTER(I32), C.POINTER(I32)]),
    "mc_scene_ingest_host": (I32, [P, P, I32, P, I32, P, P, P, C.POINTER(I32), C.POINTER(I32)]),
    "mc_env_create": (I32, [P, I32, I32, C.c_float, C.c_float, C.POINTER(EnvMap)]),
    "mc_env_destroy": (I32, [C.POINTER(EnvMap)]),
    "mc_scene_generate": (I32, [C.POINTER(SceneDesc), C.POINTER(SceneHost)]),
    "mc_scene_free": (I32, [C.POINTER(SceneHost)]),
    "mc_morton_codes": (I32, [P, C.POINTER(SceneView), P, C.POINTER(AABB)]),
    "mc_radix_sort_pairs": (I32, [P, P, P, I32, I32]),
    "mc_radix_sort_pairs_static": (I32, [P, P, P, I32, I32]),
    "mc_bvh_build": (I32, [P, C.POINTER(SceneView), C.POINTER(BvhBuildOpts), C.POINTER(P)]),
    "mc_bvh_build_batch": (I32, [P, P, I32, C.POINTER(BvhBuildOpts), C.POINTER(P)]),
    "mc_bvh_export_traversal": (I32, [P, P, P]),
    "mc_render_batch": (I32, [P, P, P, I32, I32, C.POINTER(RenderStats)]),
    "mc_bvh_free": (I32, [P]),
    "mc_bvh_get_info": (I32, [P, C.POINTER(BvhInfo)]),
    "mc_bvh_export": (I32, [P, P, P, P, P, P]),
    "mc_trace_closest": (I32, [P, P, C.POINTER(SceneView), P, I32, I32, P]),
    "mc_trace_any": (I32, [P, P, C.POINTER(SceneView), P, P, I32, I32, P]),
    "mc_render_wavefront": (I32, [P, P, C.POINTER(SceneView), C.POINTER(RenderParams), P, C.POINTER(RenderStats)]),
    "mc_render_host": (I32, [P, P, I32, P, I32, C.POINTER(EnvMap), C.POINTER(RenderParams), P, C.POINTER(RenderStats)]),
    "mc_rng_reset": (I32, [P, I32, I32, C.c_uint64]),
    "mc_autotune": (I32, [P, P, C.POINTER(SceneView), C.POINTER(RenderParams), I32]),
    "mc_guide_create": (I32, [P, C.POINTER(GuideConfig), C.POINTER(P)]),
    "mc_guide_destroy": (I32, [P]),
    "mc_guide_get_params": (I32, [P, P]),
    "mc_guide_set_params": (I32, [P, P]),
    "mc_guide_infer": (I32, [P, P, I32, P]),
    "mc_guide_gradient": (I32, [P, P, I32, P, C.POINTER(C.c_double)]),
    "mc_guide_train": (I32, [P, P, I32]),
    "mc_guide_steps": (I32, [P]),
    "mc_render_guided": (I32, [P, P, C.POINTER(SceneView), C.POINTER(RenderParams), P, I32, P,
                               C.POINTER(RenderStats)]),
    "mc_server_create": (I32, [P, C.POINTER(ServerConfig), C.POINTER(P)]),
    "mc_server_destroy": (I32, [P]),
    "mc_server_add_scene": (I32, [P, C.POINTER(SceneView), C.POINTER(C.c_int64)]),
    "mc_server_submit": (I32, [P, C.POINTER(ServerRequest), C.POINTER(C.c_int64)]),
    "mc_server_step": (I32, [P, C.POINTER(I32)]),
    "mc_server_get_result": (I32, [P, C.c_int64, C.POINTER(ServerResult)]),
    "mc_server_release": (I32, [P, C.c_int64]),
    "mc_server_cancel": (I32, [P, C.c_int64]),
    "mc_server_read": (I32, [P, C.c_int64, P]),
    "mc_server_encode": (I32, [P, C.c_int64, C.POINTER(ImageOptions), P, C.POINTER(C.c_int64), C.POINTER(C.c_float)]),
    "mc_image_encode": (I32, [P, P, I32, I32, I32, C.POINTER(ImageOptions), P, C.POINTER(C.c_int64),
                              C.POINTER(C.c_float)]),
    "mc_png_encode": (I32, [P, I32, I32, P, C.POINTER(C.c_int64)]),
    "mc_obj_load": (I32, [C.c_char_p, C.POINTER(Material), Vec3, C.c_float, C.c_float, I32, C.POINTER(SceneHost),
                          C.POINTER(ObjInfo)]),
    "mc_obj_info_free": (I32, [C.POINTER(ObjInfo)]),
    "mc_ppm_read": (I32, [C.c_char_p, C.POINTER(I32), C.POINTER(I32), P]),
    "mc_image_texture_create": (I32, [P, I32, I32, C.POINTER(C.c_uint64)]),
    "mc_image_texture_destroy": (I32, [C.c_uint64]),
    "mc_image_encode_host": (I32, [P, P, I32, I32, I32, C.POINTER(ImageOptions), P, C.POINTER(C.c_int64),
                                   C.POINTER(C.c_float)]),
    "mc_volume_grid_create": (I32, [P, P, I32, I32, I32, P, C.c_float, C.POINTER(C.c_void_p), C.POINTER(VolumeGrid)]),
    "mc_volume_grid_destroy": (I32, [P]),
    "mc_volume_fog_sphere": (I32, [C.c_float, C.c_float, C.c_float, P, P, P]),
    "mc_volume_density": (I32, [P, P, P, I32, P]),
    "mc_volume_file_read": (I32, [C.c_char_p, P, P, C.POINTER(C.c_float), P]),
    "mc_volume_file_write": (I32, [C.c_char_p, P, P, C.c_float, P]),
    "mc_pfm_read": (I32, [C.c_char_p, C.POINTER(I32), C.POINTER(I32), P]),
    "mc_scene_cloud": (I32, [P, C.POINTER(VolumeGrid), I32, C.POINTER(SceneHost)]),
    "mc_server_get_stats": (I32, [P, C.POINTER(ServerStats)]),
    "mc_server_now": (C.c_double, [P]),
}

_lib = None


def load(path=None):
    """Loads libmcpt.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("MCPT_LIBRARY") or LIB_PATH
    if not os.path.exists(path):
        raise McError(10, "libmcpt.so not built (run monocuda-pt_b200/build.py): %s" % path)
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status):
    if status != MC_OK:
        msg = load().mc_last_error()
        raise McError(status, msg.decode() if msg else "")
    return status


def ptr(x):
    """Device/host address of a torch tensor, numpy array, ctypes object or int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    return C.addressof(x)


class Context:
    def __init__(self, device=0):
        self.lib = load()
        h = P()
        check(self.lib.mc_context_create(device, C.byref(h)))
        self.handle = h

    def set_stream(self, stream_ptr):
        check(self.lib.mc_context_set_stream(self.handle, stream_ptr))

    def synchronize(self):
        check(self.lib.mc_context_synchronize(self.handle))

    def close(self):
        if self.handle:
            self.lib.mc_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Bvh:
    def __init__(self, ctx, view, permutation=None, layout=LAYOUT_BINARY, keep_reference_nodes=False,
                 builder=BUILDER_CLUSTERED, phase_launches=False):
        self.ctx = ctx
        self.lib = ctx.lib
        opts = BvhBuildOpts(ptr(permutation), layout, 1 if keep_reference_nodes else 0, builder,
                            1 if phase_launches else 0)
        h = P()
        check(self.lib.mc_bvh_build(ctx.handle, C.byref(view), C.byref(opts), C.byref(h)))
        self.handle = h

    def info(self):
        i = BvhInfo()
        check(self.lib.mc_bvh_get_info(self.handle, C.byref(i)))
        return i

    def export(self, codes=None, ids=None, types=None, internal=None, leaves=None):
        check(self.lib.mc_bvh_export(self.handle, ptr(codes), ptr(ids), ptr(types), ptr(internal), ptr(leaves)))

    def traversal_arrays(self):
        """The node array and the leaf-ordered primitive records the traversal
        reads, as device uint8 tensors (mc_bvh_export_traversal)."""
        return traversal_arrays(self.lib, self.handle)

    def close(self):
        if self.handle:
            self.lib.mc_bvh_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def traversal_arrays(lib, handle):
    import torch
    i = BvhInfo()
    check(lib.mc_bvh_get_info(handle, C.byref(i)))
    nodes = torch.empty(int(i.node_bytes), dtype=torch.uint8, device="cuda")
    prims = torch.empty(int(i.prim_bytes), dtype=torch.uint8, device="cuda")
    check(lib.mc_bvh_export_traversal(handle, nodes.data_ptr(), prims.data_ptr()))
    return nodes, prims


class BatchBvh:
    """One build over several device scenes (mc_bvh_build_batch)."""

    def __init__(self, ctx, views, layout=LAYOUT_WIDE4, builder=BUILDER_CLUSTERED, phase_launches=False):
        self.ctx = ctx
        self.lib = ctx.lib
        arr = (SceneView * len(views))(*views)
        opts = BvhBuildOpts(None, layout, 0, builder, 1 if phase_launches else 0)
        h = P()
        check(self.lib.mc_bvh_build_batch(ctx.handle, C.addressof(arr), len(views), C.byref(opts), C.byref(h)))
        self.handle = h
        self.count = len(views)

    def render(self, items, use_graph=False):
        arr = (BatchItem * len(items))(*items)
        st = RenderStats()
        check(self.lib.mc_render_batch(self.ctx.handle, self.handle, C.addressof(arr), len(items), 1 if use_graph else 0,
                                       C.byref(st)))
        return st

    def close(self):
        if self.handle:
            self.lib.mc_bvh_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def host_triangles(scene):
    """The scene's triangle array as a ctypes array view (no copy)."""
    return (Triangle * scene.triangle_count).from_address(C.addressof(scene.triangles.contents))


def host_spheres(scene):
    """The scene's sphere array as a ctypes array view (no copy), or None."""
    if scene.sphere_count <= 0:
        return None
    return (Sphere * scene.sphere_count).from_address(C.addressof(scene.spheres.contents))


def host_env(scene):
    """The scene's environment image as a numpy (H, W, 4) view, or None."""
    if not scene.env_rgba or scene.env_width <= 0:
        return None
    import numpy as np
    n = scene.env_width * scene.env_height * 4
    buf = (C.c_float * n).from_address(C.addressof(scene.env_rgba.contents))
    return np.frombuffer(buf, dtype=np.float32).reshape(scene.env_height, scene.env_width, 4)


def _medium_flags(records, count, record_type):
    """MEDIUM_ANY when a record's material is isotropic, | MEDIUM_GRID when
    one of those has a density grid (what mc_scene_ingest reports)."""
    import numpy as np
    if not count:
        return 0
    size = C.sizeof(record_type)
    raw = np.frombuffer(records, dtype=np.uint8, count=count * size).reshape(count, size)
    mat = record_type.mat.offset
    t = mat + Material.type.offset
    g = mat + Material.density_grid.offset
    iso = raw[:, t:t + 4].copy().view(np.int32).ravel() == MAT_ISOTROPIC
    if not iso.any():
        return 0
    grid = raw[:, g:g + 8].copy().view(np.uint64).ravel() != 0
    return MEDIUM_ANY | (MEDIUM_GRID if (iso & grid).any() else 0)


class DeviceScene:
    """Uploads host triangles/spheres the way the reference's main() does
    (PT:4276-4303): hot/cold split, light list, environment texture. Device
    memory comes from torch (plumbing only); the view is an mc_scene_view.

    With a Context (`ctx`), the AoS triangles are uploaded as they are and the
    bounds, light list and split run on the device (mc_scene_ingest_host); without
    one they run on the host (mc_scene_finalize_host, mc_split_triangles_host).
    Both give the same bytes."""

    def __init__(self, triangles, spheres=None, env_rgba=None, env_intensity=1.0, env_rotation=0.0, device="cuda",
                 ctx=None):
        import numpy as np
        import torch
        lib = load()
        self.lib = lib
        n = len(triangles)
        ns = len(spheres) if spheres is not None else 0

        def up(arr, count, size):
            b = np.frombuffer(arr, dtype=np.uint8, count=max(count, 1) * size).copy()
            return torch.from_numpy(b).to(device)
        self.spheres = up(spheres, ns, 160) if ns else torch.zeros(160, dtype=torch.uint8, device=device)
        if ctx is not None:
            self.hot = torch.empty(max(n, 1) * 36, dtype=torch.uint8, device=device)
            self.cold = torch.empty(max(n, 1) * 192, dtype=torch.uint8, device=device)
            self.lights = torch.empty(max(n, 1) * 64, dtype=torch.uint8, device=device)
            nl, med = I32(), I32()
            torch.cuda.synchronize()
            check(lib.mc_scene_ingest_host(ctx.handle, C.addressof(triangles) if n else None, n,
                                           self.spheres.data_ptr() if ns else None, ns, self.hot.data_ptr(),
                                           self.cold.data_ptr(), self.lights.data_ptr(), C.byref(nl), C.byref(med)))
            self.light_count = nl.value
            self._finish(n, ns, nl.value, med.value, env_rgba, env_intensity, env_rotation)
            return
        hot = (TriangleHot * max(n, 1))()
        cold = (TriangleCold * max(n, 1))()
        tri_addr = C.addressof(triangles) if n else None
        check(lib.mc_split_triangles_host(tri_addr, n, C.addressof(hot), C.addressof(cold)))
        nl = I32()
        tcopy = (Triangle * max(n, 1))()
        if n:
            C.memmove(tcopy, triangles, C.sizeof(Triangle) * n)
        check(lib.mc_scene_finalize_host(C.addressof(tcopy), n, None, C.byref(nl)))
        lights = (Light * max(nl.value, 1))()
        check(lib.mc_scene_finalize_host(C.addressof(tcopy), n, C.addressof(lights), C.byref(nl)))
        self.light_count = nl.value

        self.hot = up(hot, n, 36)
        self.cold = up(cold, n, 192)
        self.lights = up(lights, nl.value, 64)
        medium = _medium_flags(triangles, n, Triangle) | _medium_flags(spheres, ns, Sphere)
        self._finish(n, ns, nl.value, medium, env_rgba, env_intensity, env_rotation)

    def _finish(self, n, ns, nl, medium, env_rgba, env_intensity, env_rotation):
        import numpy as np
        lib = self.lib
        self.env = EnvMap()
        if env_rgba is not None:
            e = np.ascontiguousarray(env_rgba, dtype=np.float32)
            check(lib.mc_env_create(e.ctypes.data, e.shape[1], e.shape[0], env_intensity, env_rotation, C.byref(self.env)))
        else:
            self.env.intensity = env_intensity
            self.env.rotation = env_rotation
        v = SceneView()
        v.spheres = self.spheres.data_ptr()
        v.sphere_count = ns
        v.tri_hot = self.hot.data_ptr()
        v.tri_cold = self.cold.data_ptr()
        v.triangle_count = n
        v.lights = self.lights.data_ptr()
        v.light_count = nl
        v.has_medium = int(medium)
        v.env = self.env
        self.view = v
        self.n = n + ns

    def close(self):
        if self.env.enabled:
            self.lib.mc_env_destroy(C.byref(self.env))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def volume_grid_create(ctx, density, origin, voxel_size):
    """Uploads a dense density grid, numpy (nz, ny, nx) (x fastest). Returns
    (device pointer for Material.density_grid, VolumeGrid header); the
    header's maximum_density is the Material's grid_max_density."""
    import numpy as np
    d = np.ascontiguousarray(density, dtype=np.float32)
    assert d.ndim == 3
    o = (C.c_float * 3)(*[float(x) for x in origin])
    g = C.c_void_p()
    h = VolumeGrid()
    check(load().mc_volume_grid_create(ctx.handle, d.ctypes.data, d.shape[2], d.shape[1], d.shape[0], o,
                                       float(voxel_size), C.byref(g), C.byref(h)))
    return g.value, h


def volume_grid_destroy(grid):
    check(load().mc_volume_grid_destroy(grid))


def fog_sphere(radius, voxel_size, half_width=3.0):
    """The fog sphere grid (mc_volume_fog_sphere): (density (n, n, n) float32, origin)."""
    import numpy as np
    lib = load()
    dims = (I32 * 3)()
    org = (C.c_float * 3)()
    check(lib.mc_volume_fog_sphere(radius, voxel_size, half_width, None, dims, org))
    out = np.zeros((dims[2], dims[1], dims[0]), np.float32)
    check(lib.mc_volume_fog_sphere(radius, voxel_size, half_width, out.ctypes.data, dims, org))
    return out, tuple(org)


def volume_file_write(path, density, origin, voxel_size):
    """Writes a dense grid file (mc_volume_file_write): density (nz, ny, nx)."""
    import numpy as np
    d = np.ascontiguousarray(density, dtype=np.float32)
    dims = (I32 * 3)(d.shape[2], d.shape[1], d.shape[0])
    check(load().mc_volume_file_write(path.encode(), dims, (C.c_float * 3)(*origin), float(voxel_size), d.ctypes.data))


def volume_file_read(path):
    """A dense grid file: (density (nz, ny, nx) float32, origin, voxel size)."""
    import numpy as np
    lib = load()
    dims, org, v = (I32 * 3)(), (C.c_float * 3)(), C.c_float()
    check(lib.mc_volume_file_read(path.encode(), dims, org, C.byref(v), None))
    out = np.zeros((dims[2], dims[1], dims[0]), np.float32)
    check(lib.mc_volume_file_read(path.encode(), dims, org, C.byref(v), out.ctypes.data))
    return out, tuple(org), v.value


def pfm_read(path):
    """A colour PFM as float RGBA (h, w, 4), top row first (mc_pfm_read)."""
    import numpy as np
    lib = load()
    w, h = I32(), I32()
    check(lib.mc_pfm_read(path.encode(), C.byref(w), C.byref(h), None))
    out = np.zeros((h.value, w.value, 4), np.float32)
    check(lib.mc_pfm_read(path.encode(), C.byref(w), C.byref(h), out.ctypes.data))
    return out


def volume_density(ctx, grid, d_points, n, d_out):
    """Grid values at n device points (xyz packed) into d_out, as the media sample them."""
    check(load().mc_volume_density(ctx.handle, grid, ptr(d_points), n, ptr(d_out)))


def image_encode(ctx, accum_ptr, width, height, samples, fmt=IMAGE_RGB8, tonemap=TONEMAP_NONE, exposure=1.0,
                 device_out=None):
    """Resolves and encodes a device accumulation buffer once (mc_image_encode).
    Returns (bytes or None when device_out is given, exposure applied)."""
    lib = load()
    opts = ImageOptions(fmt, tonemap, exposure, 1 if device_out is not None else 0)
    n = C.c_int64()
    check(lib.mc_image_encode(ctx.handle, accum_ptr, width, height, samples, C.byref(opts), None, C.byref(n), None))
    chosen = C.c_float()
    if device_out is not None:
        check(lib.mc_image_encode(ctx.handle, accum_ptr, width, height, samples, C.byref(opts), device_out,
                                  C.byref(n), C.byref(chosen)))
        return None, chosen.value
    buf = (C.c_uint8 * n.value)()
    check(lib.mc_image_encode(ctx.handle, accum_ptr, width, height, samples, C.byref(opts), buf, C.byref(n),
                              C.byref(chosen)))
    return bytes(buf), chosen.value


def png_encode(rgb8, width, height):
    """A PNG file (bytes) of W*H*3 8-bit RGB pixels, top row first (mc_png_encode)."""
    import numpy as np
    lib = load()
    px = np.ascontiguousarray(rgb8, dtype=np.uint8)
    n = C.c_int64()
    check(lib.mc_png_encode(None, width, height, None, C.byref(n)))
    buf = (C.c_uint8 * n.value)()
    check(lib.mc_png_encode(px.ctypes.data, width, height, buf, C.byref(n)))
    return bytes(buf)[:n.value]


def obj_load(path, fallback, translation=(0.0, 0.0, 0.0), scale=1.0, rotation_y=0.0, load_textures=False, scene=None):
    """Appends an OBJ file's triangles to a SceneHost (a new, empty one when
    scene is None) with mc_obj_load. Returns (scene, ObjInfo); free the scene
    with free_scene and the info with obj_info_free (after destroying its
    textures when the scene is no longer rendered)."""
    lib = load()
    if scene is None:
        scene = SceneHost()
    info = ObjInfo()
    check(lib.mc_obj_load(os.fsencode(path), C.byref(fallback), Vec3(*translation), scale, rotation_y,
                          1 if load_textures else 0, C.byref(scene), C.byref(info)))
    return scene, info


def obj_info_free(info, destroy_textures=True):
    lib = load()
    if destroy_textures:
        for i in range(info.textures_loaded):
            lib.mc_image_texture_destroy(info.textures[i])
    lib.mc_obj_info_free(C.byref(info))


def generate_scene(kind, variant=0, seed=0, triangle_target=0):
    """Returns a SceneHost (host memory owned by the library; free with free_scene)."""
    lib = load()
    d = SceneDesc(kind, variant, seed, triangle_target)
    s = SceneHost()
    check(lib.mc_scene_generate(C.byref(d), C.byref(s)))
    return s


def free_scene(s):
    load().mc_scene_free(C.byref(s))


def camera_initialize(cam):
    check(load().mc_camera_initialize(C.byref(cam)))
    return cam


def make_camera(width, height, look_from, look_at, vfov, focus, max_depth=8, spp=1, up=(0, 1, 0), aperture=0.0,
                background=(0, 0, 0), rr_cap=0.95):
    cam = Camera()
    cam.aspect_ratio = width / float(height)
    cam.image_width = width
    cam.samples_per_pixel = spp
    cam.max_depth = max_depth
    cam.vfov = vfov
    cam.look_from = Vec3(*look_from)
    cam.look_at = Vec3(*look_at)
    cam.up = Vec3(*up)
    cam.aperture = aperture
    cam.focus_distance = focus
    cam.background = Vec3(*background)
    cam.rr_cap = rr_cap
    return camera_initialize(cam)


def render_params(camera, width, height, spp, max_depth, persistent=True, rng=RNG_PHILOX, seed=1234, first_sample=0,
                  intersector=ISECT_REFERENCE, disable_clamp=False, refill_threshold=0, use_graph=False, instrument=0,
                  samples_per_wave=0, env_sampling=0, queue_capacity=0, stack_entries=0, trace_threads=0):
    p = RenderParams()
    p.camera = camera
    p.width, p.height, p.spp, p.first_sample, p.max_depth = width, height, spp, first_sample, max_depth
    p.persistent = 1 if persistent else 0
    p.rng = rng
    p.seed = seed
    p.intersector = intersector
    p.disable_clamp = 1 if disable_clamp else 0
    p.queue_capacity = queue_capacity
    p.refill_threshold = refill_threshold
    p.use_graph = 1 if use_graph else 0
    p.instrument = instrument
    p.samples_per_wave = samples_per_wave
    p.env_sampling = env_sampling
    p.stack_entries = stack_entries
    p.trace_threads = trace_threads
    return p


class Guide:
    """The path-guiding MLP (mc_guide_*): FP32 master weights on the device,
    BF16 tensor-core inference and training."""

    def __init__(self, ctx, bounds_lo, bounds_hi, seed=1, learning_rate=1e-3, batch_capacity=0, guide_fraction=0.5,
                 train_steps=1, train_vertices=0, direction_input=0, guided_depth=0, weight_cap=0.0, fold_below=False,
                 anchor_lobes=None, nee_records=False):
        self.ctx = ctx
        self.lib = ctx.lib
        cfg = GuideConfig()
        cfg.bounds.lo = Vec3(*bounds_lo)
        cfg.bounds.hi = Vec3(*bounds_hi)
        cfg.learning_rate = learning_rate
        cfg.seed = seed
        cfg.batch_capacity = batch_capacity
        cfg.guide_fraction = guide_fraction
        cfg.train_steps = train_steps
        cfg.train_vertices = train_vertices
        cfg.direction_input = direction_input
        cfg.guided_depth = guided_depth
        cfg.weight_cap = weight_cap
        cfg.fold_below = 1 if fold_below else 0
        # None: the library default (anchored); True / False: anchored / raw means
        cfg.anchor_lobes = 0 if anchor_lobes is None else (GUIDE_LOBES_ANCHORED if anchor_lobes else GUIDE_LOBES_RAW)
        cfg.nee_records = 1 if nee_records else 0
        self.config = cfg
        h = P()
        check(self.lib.mc_guide_create(ctx.handle, C.byref(cfg), C.byref(h)))
        self.handle = h

    def box(self):
        """(lo, 1/extent) as the kernels form them (float32)."""
        import numpy as np
        lo = np.array([self.config.bounds.lo.x, self.config.bounds.lo.y, self.config.bounds.lo.z], np.float32)
        hi = np.array([self.config.bounds.hi.x, self.config.bounds.hi.y, self.config.bounds.hi.z], np.float32)
        ext = hi - lo
        inv = np.where(ext > 0, np.float32(1.0) / np.where(ext > 0, ext, np.float32(1)), np.float32(1)).astype(np.float32)
        return lo, inv

    def get_params(self):
        import numpy as np
        out = np.zeros(GUIDE_PARAM_COUNT, np.float32)
        check(self.lib.mc_guide_get_params(self.handle, out.ctypes.data))
        return out

    def set_params(self, params):
        import numpy as np
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == GUIDE_PARAM_COUNT
        check(self.lib.mc_guide_set_params(self.handle, p.ctypes.data))

    def steps(self):
        return self.lib.mc_guide_steps(self.handle)

    def close(self):
        if self.handle:
            self.lib.mc_guide_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The render server (mc_server_*): resident scenes, HBM-budget admission,
    shared waves for all active requests."""

    def __init__(self, ctx, budget_bytes=0, max_active=0, samples_per_step=0, wave_paths=0, flags=0):
        self.ctx = ctx
        self.lib = ctx.lib
        cfg = ServerConfig(budget_bytes, max_active, samples_per_step, wave_paths, flags, 0)
        h = P()
        check(self.lib.mc_server_create(ctx.handle, C.byref(cfg), C.byref(h)))
        self.handle = h
        self.views = []  # the scene views must outlive the server

    def add_scene(self, device_scene):
        sid = C.c_int64()
        check(self.lib.mc_server_add_scene(self.handle, C.byref(device_scene.view), C.byref(sid)))
        self.views.append(device_scene)
        return sid.value

    def submit(self, scene_id, params, guided=False):
        req = ServerRequest(scene_id, params, 1 if guided else 0)
        rid = C.c_int64()
        check(self.lib.mc_server_submit(self.handle, C.byref(req), C.byref(rid)))
        return rid.value

    def step(self):
        a = I32()
        check(self.lib.mc_server_step(self.handle, C.byref(a)))
        return a.value

    def result(self, rid):
        r = ServerResult()
        check(self.lib.mc_server_get_result(self.handle, rid, C.byref(r)))
        return r

    def read(self, rid, width, height):
        """The request's accumulation buffer (sum over its samples) as a host array."""
        import numpy as np
        out = np.zeros(width * height * 3, np.float32)
        check(self.lib.mc_server_read(self.handle, rid, out.ctypes.data))
        return out

    def encode(self, rid, fmt=IMAGE_RGB8, tonemap=TONEMAP_NONE, exposure=1.0):
        """The request's image encoded once (mc_server_encode): bytes, and the
        exposure applied (exposure <= 0: automatic)."""
        opts = ImageOptions(fmt, tonemap, exposure, 0)
        n = C.c_int64()
        check(self.lib.mc_server_encode(self.handle, rid, C.byref(opts), None, C.byref(n), None))
        buf = (C.c_uint8 * n.value)()
        chosen = C.c_float()
        check(self.lib.mc_server_encode(self.handle, rid, C.byref(opts), buf, C.byref(n), C.byref(chosen)))
        return bytes(buf), chosen.value

    def release(self, rid):
        check(self.lib.mc_server_release(self.handle, rid))

    def cancel(self, rid):
        check(self.lib.mc_server_cancel(self.handle, rid))

    def stats(self):
        st = ServerStats()
        check(self.lib.mc_server_get_stats(self.handle, C.byref(st)))
        return st

    def now(self):
        return self.lib.mc_server_now(self.handle)

    def close(self):
        if self.handle:
            self.lib.mc_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
